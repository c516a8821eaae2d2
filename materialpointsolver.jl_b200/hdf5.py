"""HDF5 snapshot files without libhdf5.

``H5File`` wraps the library's writer (``mpm_h5_*`` in include/mpm_b200.h),
which produces the tree submit_work! writes through HDF5.jl
(src/solver.jl:54-111): ``group<i>/{stress, strain_s, eqstrain, ekstrain,
eqrate, coords, velocity_s, volume, mass_s, time}`` per snapshot, then
``FILE_NUM``, ``grid_coords``, ``mp_coords0``, ``nid`` and ``vbc_*`` at the root.

Arrays are given in the reference's layout (a Julia ``n x k`` matrix is a
numpy ``(n, k)`` array); like HDF5.jl, the file stores it as the dataspace
``(k, n)`` over the column-major buffer, so h5py reads it back as ``(k, n)``
and HDF5.jl as ``n x k``.

``read`` parses the subset of the format the writer emits (superblock 0,
version-1 object headers, symbol-table groups, contiguous datasets) into
nested dicts of numpy arrays, checking the structural rules of the format
on the way (signatures, member order, B-tree keys, end-of-file address).
"""
from __future__ import annotations

import ctypes as C
import struct

import numpy as np

from . import _lib

_TYPES = {np.dtype(np.float64): _lib.T_F64, np.dtype(np.float32): _lib.T_F32,
          np.dtype(np.int64): _lib.T_I64, np.dtype(np.int32): _lib.T_I32}


class H5File:
    """An HDF5 file being written; readable once ``close()`` returned."""

    def __init__(self, path):
        self.path = str(path)
        h = C.c_void_p()
        _lib.check(_lib.lib().mpm_h5_create(self.path.encode(), C.byref(h)))
        self.h = h

    def write(self, name, a):
        """Dataset ``name`` ("group1/stress") from a scalar, a vector or an
        ``(n, k)`` matrix in the reference's layout."""
        a = np.asarray(a)
        if a.dtype == np.bool_:
            a = a.astype(np.int64)
        if a.dtype not in _TYPES:
            a = a.astype(np.float64 if a.dtype.kind == "f" else np.int64)
        if a.ndim > 2:
            raise ValueError("datasets of rank 0, 1 or 2")
        buf = np.asfortranarray(a) if a.ndim == 2 else np.ascontiguousarray(a)
        dims = (C.c_int64 * 2)(*(reversed(a.shape) if a.ndim == 2 else a.shape + (0,) * (2 - a.ndim)))
        _lib.check(_lib.lib().mpm_h5_write(self.h, name.encode(), _TYPES[a.dtype], a.ndim, dims,
                                           buf.ctypes.data if buf.size else None))

    def close(self):
        if self.h:
            h, self.h = self.h, None
            _lib.check(_lib.lib().mpm_h5_close(h))

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


# ---- reader ------------------------------------------------------------------------

_UNDEF = (1 << 64) - 1


def _u(b, off, n):
    return int.from_bytes(b[off:off + n], "little")


def _messages(b, addr):
    if b[addr] != 1:
        raise ValueError(f"object header at {addr}: version {b[addr]} (expected 1)")
    nmsg, size = _u(b, addr + 2, 2), _u(b, addr + 8, 4)
    p, end, out = addr + 16, addr + 16 + size, []
    while p < end:
        t, sz = _u(b, p, 2), _u(b, p + 2, 2)
        if sz % 8:
            raise ValueError(f"object header at {addr}: message size {sz} not 8-byte aligned")
        out.append((t, b[p + 8:p + 8 + sz]))
        p += 8 + sz
    if p != end or len(out) != nmsg:
        raise ValueError(f"object header at {addr}: {len(out)} messages, header says {nmsg}")
    return dict(out)


def _dataset(b, msgs):
    sp, dt, lay = msgs[0x0001], msgs[0x0003], msgs[0x0008]
    if sp[0] != 1:
        raise ValueError("dataspace version")
    rank = sp[1]
    dims = tuple(_u(sp, 8 + 8 * r, 8) for r in range(rank))
    cls, ver, size = dt[0] & 0x0F, dt[0] >> 4, _u(dt, 4, 4)
    if ver != 1 or dt[1] & 1:
        raise ValueError("datatype version / byte order")
    if cls == 1:
        prec, eloc, esz, mloc, msz, bias = struct.unpack_from("<xxHBBBBI", dt, 8)
        ref = {8: (64, 52, 11, 0, 52, 1023), 4: (32, 23, 8, 0, 23, 127)}[size]
        if (prec, eloc, esz, mloc, msz, bias) != ref or dt[2] != 8 * size - 1:
            raise ValueError("non-IEEE floating-point type")
        dtype = np.dtype(f"<f{size}")
    elif cls == 0:
        dtype = np.dtype(f"<{'i' if dt[1] & 0x08 else 'u'}{size}")
    else:
        raise ValueError(f"datatype class {cls}")
    if lay[0] != 3 or lay[1] != 1:
        raise ValueError("only contiguous layout (version 3)")
    addr, nbytes = _u(lay, 2, 8), _u(lay, 10, 8)
    n = int(np.prod(dims)) if rank else 1
    if nbytes != n * dtype.itemsize:
        raise ValueError("layout size does not match the dataspace")
    if n == 0:
        return np.zeros(dims, dtype)
    a = np.frombuffer(b, dtype, count=n, offset=addr).reshape(dims) if rank else \
        np.frombuffer(b, dtype, count=1, offset=addr)[0]
    return a.copy()


def _group(b, addr, leaf_k, int_k):
    msgs = _messages(b, addr)
    stab = msgs[0x0011]
    bt, hp = _u(stab, 0, 8), _u(stab, 8, 8)
    if b[hp:hp + 4] != b"HEAP" or b[hp + 4] != 0:
        raise ValueError(f"local heap at {hp}")
    dsize, free, data = _u(b, hp + 8, 8), _u(b, hp + 16, 8), _u(b, hp + 24, 8)
    if free != 1 and free >= dsize:
        raise ValueError("local heap free list")
    heap = b[data:data + dsize]

    def name(off):
        return heap[off:heap.index(b"\0", off)].decode()

    if b[bt:bt + 4] != b"TREE" or b[bt + 4] != 0 or b[bt + 5] != 0:
        raise ValueError(f"group B-tree at {bt}: only a leaf-level group node is read")
    n = _u(b, bt + 6, 2)
    if n > 2 * int_k:
        raise ValueError("B-tree node over capacity")
    p = bt + 24
    keys, kids = [name(_u(b, p, 8))], []
    p += 8
    for _ in range(n):
        kids.append(_u(b, p, 8))
        keys.append(name(_u(b, p + 8, 8)))
        p += 16
    if keys[0] != "":
        raise ValueError("left-most B-tree key must be the empty name")
    out, prev = {}, None
    for i, sn in enumerate(kids):
        if b[sn:sn + 4] != b"SNOD" or b[sn + 4] != 1:
            raise ValueError(f"symbol table node at {sn}")
        cnt = _u(b, sn + 6, 2)
        if cnt > 2 * leaf_k:
            raise ValueError("symbol table node over capacity")
        for j in range(cnt):
            e = sn + 8 + 40 * j
            nm, oh = name(_u(b, e, 8)), _u(b, e + 8, 8)
            if prev is not None and not nm > prev:
                raise ValueError("group members out of order")
            if not keys[i] < nm <= keys[i + 1]:
                raise ValueError("B-tree keys do not bracket the members")
            prev = nm
            m = _messages(b, oh)
            out[nm] = _group(b, oh, leaf_k, int_k) if 0x0011 in m else _dataset(b, m)
        if cnt and name(_u(b, sn + 8 + 40 * (cnt - 1), 8)) != keys[i + 1]:
            raise ValueError("B-tree key is not the last member of its child")
    return out


def read(path):
    """The tree of an HDF5 file written by ``H5File`` as nested dicts."""
    with open(path, "rb") as fh:
        b = fh.read()
    if b[:8] != b"\x89HDF\r\n\x1a\n":
        raise ValueError("not an HDF5 file")
    if b[8] != 0 or b[13] != 8 or b[14] != 8:
        raise ValueError("superblock version 0 with 8-byte offsets and lengths expected")
    leaf_k, int_k = _u(b, 16, 2), _u(b, 18, 2)
    base, eof = _u(b, 24, 8), _u(b, 40, 8)
    if base != 0 or eof != len(b):
        raise ValueError(f"end-of-file address {eof} != file size {len(b)}")
    root = _u(b, 64, 8)
    if _u(b, 72, 4) == 1:
        stab = _messages(b, root)[0x0011]
        if (_u(b, 80, 8), _u(b, 88, 8)) != (_u(stab, 0, 8), _u(stab, 8, 8)):
            raise ValueError("root entry cache disagrees with the root group")
    return _group(b, root, leaf_k, int_k)
