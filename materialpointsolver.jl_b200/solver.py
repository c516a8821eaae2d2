"""Host driver: the reference's entry point and device boundary over the C ABI.

``materialpointsolver(args, grid, mp, attr, bc)`` mirrors ``materialpointsolver!``
(src/MaterialPointSolver.jl:61-76) and ``submit_work!`` (src/solver.jl:37-131)
for ``args.device == "B200"``: upload once (host2device), advance
``while Ti < Ttol`` with the step workflow, download the fields device2host!
copies, free the device.  The per-step workflow is ``procedure`` (the
``procedure!`` of src/solvers/OS_MUSL.jl:12-102); the driver hands the device
runs of consecutive steps so the host is not in the loop of every step.
"""
from __future__ import annotations

import ctypes as C
import os
import time

import numpy as np

from . import _lib
from .types import Grid3D


def _view(a, typ=None):
    v = _lib.View()
    if a is None:
        v.ptr = None
        return v
    if not (a.flags["F_CONTIGUOUS"] or a.ndim == 1):
        raise ValueError("host arrays must be column-major (Fortran order)")
    t = {np.dtype(np.float64): _lib.T_F64, np.dtype(np.float32): _lib.T_F32,
         np.dtype(np.int64): _lib.T_I64, np.dtype(np.int32): _lib.T_I32}[a.dtype]
    v.ptr = a.ctypes.data
    v.type = t
    v.ld = a.shape[0]
    return v


def host_views(grid, mp, attr, bc):
    """Views of the reference structs' arrays, in the library's layout terms."""
    hv = _lib.HostViews()
    for name in ("xi", "vs", "sig", "eps", "epsq", "epsk", "epsv", "Omega", "Omega0", "rho", "rho0", "F",
                 "ms", "sigm", "p2c"):
        setattr(hv, name, _view(getattr(mp, name)))
    hv.nid = _view(attr.nid)
    for name in ("Ks", "Gs", "c", "phi", "psi", "sigt", "Hp", "cr"):
        setattr(hv, name, _view(getattr(attr, name)))
    hv.vx_idx, hv.vx_val = _view(bc.vx_s_idx), _view(bc.vx_s_val)
    hv.vy_idx, hv.vy_val = _view(bc.vy_s_idx), _view(bc.vy_s_val)
    if grid.dim == 3:
        hv.vz_idx, hv.vz_val = _view(bc.vz_s_idx), _view(bc.vz_s_val)
    if getattr(mp, "phase", 1) == 2:
        # two-phase fields (particle.jl:103-128), Kw and k, water BC
        hv.n, hv.rhow, hv.sigw, hv.vw = _view(mp.n), _view(mp.rho_w), _view(mp.sigw), _view(mp.vw)
        hv.epsw, hv.mw = _view(mp.epsw), _view(mp.mw)
        hv.Kw, hv.kperm = _view(attr.Kw), _view(attr.k)
        for c in "xyz"[:grid.dim]:
            idx = getattr(bc, f"v{c}_w_idx", None)
            if idx is not None:
                setattr(hv, f"v{c}w_idx", _view(idx))
                setattr(hv, f"v{c}w_val", _view(getattr(bc, f"v{c}_w_val")))
    return hv


def make_desc(args, grid, mp, attr, device=0):
    d = _lib.Desc()
    d.abi_version = _lib.ABI_VERSION
    d.dim = grid.dim
    d.precision = _lib.PREC_FP64 if getattr(args, "gpu_precision", "mixed") == "fp64" else _lib.PREC_MIXED
    d.device = device
    d.np = mp.np
    d.nmat = len(attr.Es)
    d.nnx, d.nny = grid.nnx, grid.nny
    d.nnz = grid.nnz if grid.dim == 3 else 1
    d.x1, d.y1, d.dx, d.dy = grid.x1, grid.y1, grid.dx, grid.dy
    d.z1 = grid.z1 if grid.dim == 3 else 0.0
    d.dz = grid.dz if grid.dim == 3 else 1.0
    d.lpx, d.lpy = mp.dx, mp.dy
    d.lpz = mp.dz if grid.dim == 3 else 1.0
    d.constitutive = {"linearelastic": 0, "druckerprager": 1, "mohrcoulomb": 2}.get(args.constitutive, -1)
    d.va = 0 if args.va == "a" else 1
    d.mvl = int(args.MVL)
    d.mc3d = 1 if getattr(args, "mc3d", "literal") == "restated" else 0
    d.FLIP, d.PIC, d.zeta_s, d.gravity, d.Te = args.FLIP, args.PIC, args.zeta_s, args.gravity, args.Te
    d.time_f32 = 1 if args.precision == "FP32" else 0
    d.sort_every = getattr(args, "sort_every", 0)
    d.scheme = _lib.SCHEME_USL if getattr(args, "scheme", "MUSL") == "USL" else _lib.SCHEME_MUSL
    d.coupling = _lib.COUPLING_TS if getattr(args, "coupling", "OS") == "TS" else _lib.COUPLING_OS
    d.zeta_w = getattr(args, "zeta_w", 0.0)
    return d


class DeviceModel:
    """Device-resident model: the B200 counterpart of the (dev_grid, dev_mp,
    dev_attr, dev_bc) tuple host2device returns."""

    def __init__(self, args, grid, mp, attr, bc, device=0):
        L = _lib.lib()
        self.args, self.grid, self.mp, self.attr, self.bc = args, grid, mp, attr, bc
        self.desc = make_desc(args, grid, mp, attr, device)
        h = C.c_void_p()
        _lib.check(L.mpm_create(C.byref(self.desc), C.byref(h)))
        self.h = h
        self.upload()

    # host2device (devicehelpfunc_cuda.jl:17-37)
    def upload(self):
        hv = host_views(self.grid, self.mp, self.attr, self.bc)
        _lib.check(_lib.lib().mpm_upload(self.h, C.byref(hv)), self.h)

    def step(self, dt, Ti, nsteps=1):
        out = C.c_double()
        _lib.check(_lib.lib().mpm_step(self.h, dt, Ti, nsteps, C.byref(out)), self.h)
        return out.value

    def step_async(self, dt, Ti, nsteps=1):
        _lib.check(_lib.lib().mpm_step_async(self.h, dt, Ti, nsteps), self.h)

    def sync(self):
        _lib.check(_lib.lib().mpm_sync(self.h), self.h)

    # device2host! (devicehelpfunc_cuda.jl:39-69)
    def download(self, mask=_lib.F_REFERENCE, mp=None):
        mp = mp if mp is not None else self.mp
        hv = host_views(self.grid, mp, self.attr, self.bc)
        _lib.check(_lib.lib().mpm_download(self.h, C.byref(hv), mask), self.h)

    def p2c(self):
        out = np.zeros(self.mp.np, np.int64)
        _lib.check(_lib.lib().mpm_compute_p2c(self.h, out.ctypes.data_as(C.POINTER(C.c_int64))), self.h)
        return out

    def order(self):
        out = np.zeros(self.mp.np, np.int64)
        _lib.check(_lib.lib().mpm_download_order(self.h, out.ctypes.data_as(C.POINTER(C.c_int64))), self.h)
        return out

    def sort(self):
        _lib.check(_lib.lib().mpm_sort(self.h), self.h)

    def run_stages(self, dt, Ti, mask):
        _lib.check(_lib.lib().mpm_run_stages(self.h, dt, Ti, mask), self.h)

    def grid_field(self, field):
        D = self.grid.dim
        n = self.grid.ni * (1 if field == 0 else D)
        out = np.zeros(n, np.float64)
        _lib.check(_lib.lib().mpm_download_grid(self.h, field, out.ctypes.data_as(C.POINTER(C.c_double))),
                   self.h)
        return out if field == 0 else out.reshape((self.grid.ni, D), order="F")

    def stats(self):
        s = _lib.Stats()
        _lib.check(_lib.lib().mpm_get_stats(self.h, C.byref(s)), self.h)
        return s

    def set_profiling(self, on=True):
        _lib.check(_lib.lib().mpm_set_profiling(self.h, 1 if on else 0), self.h)

    def kernel_times(self):
        cap = 32
        names = (C.c_char_p * cap)()
        ms = (C.c_double * cap)()
        nl = (C.c_int64 * cap)()
        cnt = C.c_int32()
        _lib.check(_lib.lib().mpm_get_kernel_times(self.h, names, ms, nl, cap, C.byref(cnt)), self.h)
        return {names[i].decode(): (ms[i], nl[i]) for i in range(min(cnt.value, cap))}

    # run-time tuning of the step (no counterpart in the reference)
    def set_tuning(self, sort_every, tiled=0):
        """Re-sort period and particle-pass variant (0 lane-merged, 1 tiled, 2 box,
        3 lane-merged with the fused pass at 3 resident CTAs per SM)."""
        _lib.check(_lib.lib().mpm_set_tuning(self.h, int(sort_every), int(tiled)), self.h)

    def tuning(self):
        s, t = C.c_int32(), C.c_int32()
        _lib.check(_lib.lib().mpm_get_tuning(self.h, C.byref(s), C.byref(t)), self.h)
        return s.value, t.value

    def set_tile(self, tx, ty, tz=1):
        """Sort tile shape in cells (one of the compiled shapes); the next step re-sorts."""
        _lib.check(_lib.lib().mpm_set_tile(self.h, int(tx), int(ty), int(tz)), self.h)

    def tile(self):
        t = [C.c_int32() for _ in range(3)]
        _lib.check(_lib.lib().mpm_get_tile(self.h, *[C.byref(x) for x in t]), self.h)
        return tuple(x.value for x in t)

    def autotune(self, dt, Ti, steps_per_trial=32):
        """Time every (tile shape, sort period, particle-pass variant)
        candidate on real steps of this model, time the two finalists again
        back to back and keep the faster.  Returns
        (Ti after the trial steps, sort_every, variant, per-trial ms per step in
        the library's candidate order); self.tile() gives the chosen shape."""
        Tout, s, t = C.c_double(), C.c_int32(), C.c_int32()
        cap = 32
        ms = (C.c_double * cap)()
        _lib.check(_lib.lib().mpm_autotune(self.h, dt, Ti, steps_per_trial, C.byref(Tout), C.byref(s),
                                           C.byref(t), ms, cap), self.h)
        ntrial = 4 * (3 if self.grid.dim == 3 else 2) + 2 + 4 + 2
        return Tout.value, s.value, t.value, list(ms)[:ntrial]

    # stress-return surrogate (no counterpart in the reference)
    def set_surrogate(self, sur, tol=1e-3, sref=1e3):
        """Replace the 3D Drucker-Prager return by the trained surrogate `sur`
        (surrogate.Surrogate), with the yield-residual acceptance test; None
        restores the plain return."""
        if sur is None:
            _lib.check(_lib.lib().mpm_set_surrogate(self.h, None, None, 0, 0.0, 0.0, 0), self.h)
            return
        P = np.ascontiguousarray(sur.params(), np.float32)
        N = np.ascontiguousarray(sur.norm.cpu().numpy(), np.float32)
        _lib.check(_lib.lib().mpm_set_surrogate(self.h, P.ctypes.data, N.ctypes.data, sur.flags, float(tol),
                                                float(sref), 1), self.h)

    def log_samples(self, feat, target, count, every):
        """Log training samples of the plain return into device tensors
        (feat: cap x 16, target: cap x 6 FP32, count: 1 int32); every = 0 stops."""
        if every == 0:
            _lib.check(_lib.lib().mpm_log_samples(self.h, None, None, None, 0, 0), self.h)
            return
        cap = min(feat.shape[0], target.shape[0])
        _lib.check(_lib.lib().mpm_log_samples(self.h, feat.data_ptr(), target.data_ptr(), count.data_ptr(), cap,
                                              int(every)), self.h)

    # HDF5 snapshots (submit_work!, src/solver.jl:60-76)
    def snapshot(self, h5file, group, Ti, fields=_lib.F_SNAPSHOT, dtype=np.float64):
        """Enqueue group ``group<group>`` of the particle fields and ``time`` =
        Ti into ``h5file`` (hdf5.H5File); returns at once, the copy and the
        file write overlap the following steps."""
        t = _lib.T_F64 if np.dtype(dtype) == np.float64 else _lib.T_F32
        _lib.check(_lib.lib().mpm_snapshot(self.h, h5file.h, int(group), float(Ti), fields, t), self.h)

    def snapshot_wait(self):
        """Wait until every enqueued snapshot is in its file; returns how many
        groups were written."""
        n = C.c_int64()
        _lib.check(_lib.lib().mpm_snapshot_wait(self.h, C.byref(n)), self.h)
        return n.value

    # clean_device! (devicehelpfunc_cuda.jl:71-100)
    def close(self):
        if getattr(self, "h", None):
            _lib.lib().mpm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def host2device(args, grid, mp, attr, bc, device=0):
    return DeviceModel(args, grid, mp, attr, bc, device)


def device2host(args, mp, dev, verbose=False):
    dev.download(_lib.F_REFERENCE_TS if args.coupling == "TS" else _lib.F_REFERENCE, mp)
    if verbose:
        print("downloading from :B200 -> host")


def clean_device(dev):
    dev.close()


def time_sequence(args, Ti0=0.0):
    """Ti values of submit_work!'s loop (src/solver.jl:118-125): `while Ti < Ttol;
    …; Ti += ΔT` with Ti in the model's float type T2."""
    f32 = args.precision == "FP32"
    T = np.float32 if f32 else np.float64
    Ti, dt, Ttol = T(Ti0), T(args.dT), T(args.Ttol)
    n = 0
    while Ti < Ttol:
        Ti = T(Ti + dt)
        n += 1
    return n


def procedure(args, dev, dT, Ti):
    """One step, the B200 counterpart of procedure!(…, Val(:OS), Val(:MUSL), Val(va))."""
    dev.step(dT, Ti, 1)


def snapshot_path(args):
    """<project_path>/<project_name>/<project_name>.h5 (src/solver.jl:57)."""
    return os.path.join(args.project_path, args.project_name, f"{args.project_name}.h5")


def _run_with_snapshots(args, grid, mp, attr, bc, dev, nsteps, workflow):
    """submit_work!'s HDF5 branch (src/solver.jl:54-111): a group before the
    step whenever ``hdf5_switch`` is 0 or ``hdf5_step``, i.e. before steps 0,
    hdf5_step, 2*hdf5_step, ...; then FILE_NUM (groups written + 1), the grid
    coordinates, the initial particle coordinates, nid and the velocity BCs.
    The runs between snapshots go to the device as one call; each snapshot's
    copy and file write overlap the next run."""
    from .hdf5 import H5File
    T = np.float32 if args.precision == "FP32" else np.float64
    path = snapshot_path(args)
    if os.path.isfile(path):
        os.remove(path)
    os.makedirs(os.path.dirname(path), exist_ok=True)
    f = H5File(path)
    try:
        hdf5_id, done, Ti = 1, 0, T(0.0)
        fields = _lib.F_SNAPSHOT_TS if args.coupling == "TS" else _lib.F_SNAPSHOT
        while done < nsteps:
            dev.snapshot(f, hdf5_id, float(Ti), fields=fields, dtype=T)
            hdf5_id += 1
            n = min(args.hdf5_step, nsteps - done)
            if workflow is None:
                Ti = T(dev.step(args.dT, float(Ti), n))
            else:
                for _ in range(n):
                    workflow(args, dev, args.dT, float(Ti))
                    Ti = T(Ti + T(args.dT))
            done += n
        dev.snapshot_wait()
        I = attr.nid.dtype
        f.write("FILE_NUM", np.asarray(hdf5_id, I))
        f.write("grid_coords", grid.xi)
        f.write("mp_coords0", mp.xi0)
        f.write("nid", attr.nid)
        axes = ("x", "y", "z")[:grid.dim]
        for a in axes:
            f.write(f"vbc_{a}s_idx", getattr(bc, f"v{a}_s_idx"))
            f.write(f"vbc_{a}s_val", getattr(bc, f"v{a}_s_val"))
        if args.coupling == "TS":
            for a in axes:
                f.write(f"vbc_{a}w_idx", getattr(bc, f"v{a}_w_idx"))
                f.write(f"vbc_{a}w_val", getattr(bc, f"v{a}_w_val"))
    finally:
        try:
            dev.snapshot_wait()
        finally:
            f.close()


def materialpointsolver(args, grid, mp, attr, bc, workflow=None, device=0, verbose=False):
    """Entry point mirroring materialpointsolver! (src/MaterialPointSolver.jl:61-76).

    ``workflow=None`` runs the library's step for all steps in one device call;
    a callable ``workflow(args, dev, dT, Ti)`` is called once per step instead,
    like the reference's ``workflow`` keyword."""
    if args.device != "B200":
        raise ValueError("this package provides the :B200 device backend (args.device = 'B200')")
    if not ((args.coupling == "OS" and args.scheme in ("MUSL", "USL")) or
            (args.coupling == "TS" and args.scheme == "MUSL")):
        raise NotImplementedError("the one-phase MUSL and USL and the two-phase MUSL schemes are provided")
    if args.basis != "uGIMP":
        raise NotImplementedError("only the uGIMP basis is provided")
    dev = host2device(args, grid, mp, attr, bc, device)
    try:
        mp.p2c[:] = dev.p2c().astype(mp.p2c.dtype)   # initmpstatus! (src/solver.jl:45)
        nsteps = time_sequence(args)
        args.start_time = time.time()
        if args.hdf5:
            _run_with_snapshots(args, grid, mp, attr, bc, dev, nsteps, workflow)
        elif workflow is None:
            Ti = dev.step(args.dT, 0.0, nsteps) if nsteps else 0.0
        else:
            T = np.float32 if args.precision == "FP32" else np.float64
            Ti = T(0.0)
            for _ in range(nsteps):
                workflow(args, dev, args.dT, float(Ti))
                Ti = T(Ti + T(args.dT))
        args.end_time = time.time()
        args.iter_num += nsteps
        device2host(args, mp, dev, verbose=verbose)
    finally:
        clean_device(dev)
    if verbose:
        dtw = args.end_time - args.start_time
        print(f"wall time {dtw:.3f} s, {nsteps} iterations, {nsteps / max(dtw, 1e-12):.3e} it/s")
    return None
