"""HDF5 snapshots (the output branch of submit_work!, src/solver.jl:54-111).

CPU: the library's HDF5 writer (mpm_h5_*) round-trips datasets of every
element type and rank through the format reader, lays the file out as the
format requires (superblock fields, end-of-file address, node sizes from the
superblock's K values, member order), rejects bad input; the host loop takes
its snapshots before the steps submit_work! takes them and writes the root
datasets (a stand-in device records the calls).

GPU: every group holds exactly what a download of the same device state
returns (FP64 and FP32 models); materialpointsolver with hdf5 = true writes
one group per hdf5_step steps that matches a second model stepped by the same
chunks, to the run-to-run spread of the floating-point reductions."""
import math
import os

import numpy as np
import pytest

from helpers import fresh_particles, rel


def _h5(pkg):
    return pkg.hdf5


def test_roundtrip_types_and_ranks(pkg, tmp_path):
    h5 = _h5(pkg)
    rng = np.random.default_rng(3)
    A = rng.standard_normal((37, 6))            # a Julia 37 x 6 matrix
    B = rng.standard_normal((37, 3)).astype(np.float32)
    I64 = rng.integers(-2**40, 2**40, 11)
    I32 = rng.integers(-2**30, 2**30, 5).astype(np.int32)
    p = tmp_path / "a.h5"
    with h5.H5File(p) as f:
        f.write("group1/stress", A)
        f.write("group1/velocity_s", B)
        f.write("group1/time", np.float64(0.125))
        f.write("group1/t32", np.float32(0.5))
        f.write("nid", I64)
        f.write("small", I32)
        f.write("FILE_NUM", np.int64(2))
        f.write("empty", np.zeros(0))
        f.write("a/b/c/deep", np.arange(4.0))
    t = h5.read(p)
    assert set(t) == {"group1", "nid", "small", "FILE_NUM", "empty", "a"}
    g = t["group1"]
    # HDF5.jl's convention: the dataspace of an n x k matrix is (k, n)
    assert g["stress"].shape == (6, 37) and np.array_equal(g["stress"].T, A)
    assert g["velocity_s"].dtype == np.float32 and np.array_equal(g["velocity_s"].T, B)
    assert g["time"] == 0.125 and g["time"].dtype == np.float64
    assert g["t32"] == 0.5 and g["t32"].dtype == np.float32
    assert np.array_equal(t["nid"], I64) and t["nid"].dtype == np.int64
    assert np.array_equal(t["small"], I32) and t["small"].dtype == np.int32
    assert t["FILE_NUM"] == 2
    assert t["empty"].shape == (0,)
    assert np.array_equal(t["a"]["b"]["c"]["deep"], np.arange(4.0))


def _u(b, off, n):
    return int.from_bytes(b[off:off + n], "little")


@pytest.mark.parametrize("ngroups", [1, 9, 130, 700])
def test_file_layout(pkg, tmp_path, ngroups):
    """Superblock 0 fields, EOF address, leaf K sized so one B-tree node
    addresses every member, B-tree and symbol-table nodes allocated at the
    sizes a reader derives from the superblock's K values."""
    h5 = _h5(pkg)
    p = tmp_path / "b.h5"
    with h5.H5File(p) as f:
        for i in range(1, ngroups + 1):
            f.write(f"group{i}/time", np.float64(i))
    b = open(p, "rb").read()
    assert b[:8] == b"\x89HDF\r\n\x1a\n"
    assert list(b[8:16]) == [0, 0, 0, 0, 0, 8, 8, 0]
    leaf_k, int_k = _u(b, 16, 2), _u(b, 18, 2)
    assert int_k == 16 and leaf_k == max(4, math.ceil(ngroups / 64))
    assert _u(b, 20, 4) == 0 and _u(b, 24, 8) == 0
    assert _u(b, 32, 8) == 2**64 - 1 and _u(b, 48, 8) == 2**64 - 1
    assert _u(b, 40, 8) == len(b)
    assert _u(b, 72, 4) == 1                      # root entry caches B-tree and heap
    bt, heap = _u(b, 80, 8), _u(b, 88, 8)
    assert b[bt:bt + 4] == b"TREE" and b[heap:heap + 4] == b"HEAP"
    assert _u(b, heap + 16, 8) == 1               # free list: none
    nsnod = _u(b, bt + 6, 2)
    assert nsnod == math.ceil(ngroups / (2 * leaf_k))
    for s in range(nsnod):
        sn = _u(b, bt + 24 + 8 + 16 * s, 8)
        assert b[sn:sn + 4] == b"SNOD"
        # the node is allocated at full capacity (8 + 2K entries of 40 bytes)
        assert sn + 8 + 2 * leaf_k * 40 <= len(b)
    assert bt + 24 + (2 * int_k + 1) * 8 + 2 * int_k * 8 <= len(b)
    t = h5.read(p)
    assert sorted(t) == sorted(f"group{i}" for i in range(1, ngroups + 1))
    assert all(t[f"group{i}"]["time"] == i for i in range(1, ngroups + 1))


def test_writer_rejects_bad_input(pkg, tmp_path):
    h5 = _h5(pkg)
    L = pkg._lib
    f = h5.H5File(tmp_path / "c.h5")
    f.write("x", np.zeros(3))
    with pytest.raises(L.MPMError, match="exists"):
        f.write("x", np.zeros(3))
    with pytest.raises(L.MPMError, match="bad dataset path"):
        f.write("x/y", np.zeros(3))                # through a dataset
    with pytest.raises(L.MPMError, match="bad dataset path"):
        f.write("g//y", np.zeros(3))
    with pytest.raises(ValueError):
        f.write("r3", np.zeros((2, 2, 2)))
    f.close()
    f.close()                                      # idempotent
    with pytest.raises(L.MPMError, match="cannot create"):
        h5.H5File(tmp_path / "no_such_dir" / "d.h5")


def test_reader_rejects_a_truncated_file(pkg, tmp_path):
    h5 = _h5(pkg)
    p = tmp_path / "e.h5"
    with h5.H5File(p) as f:
        f.write("v", np.arange(10.0))
    b = open(p, "rb").read()
    open(p, "wb").write(b[:-8])
    with pytest.raises(ValueError, match="end-of-file"):
        h5.read(p)


class _FakeDevice:
    """Stands in for DeviceModel: records the snapshot schedule and writes
    the host arrays as the group."""

    def __init__(self, mp):
        self.mp, self.calls, self.steps = mp, [], 0

    def snapshot(self, f, group, Ti, fields=None, dtype=np.float64):
        self.calls.append((group, self.steps, Ti))
        f.write(f"group{group}/coords", self.mp.xi)
        f.write(f"group{group}/time", np.asarray(Ti, dtype))

    def step(self, dT, Ti, n):
        self.steps += n
        T = np.float32 if self.mp.xi.dtype == np.float32 else np.float64
        for _ in range(n):
            Ti = T(T(Ti) + T(dT))
        return float(Ti)

    def snapshot_wait(self):
        return len(self.calls)


@pytest.mark.parametrize("hdf5_step", [1, 7, 50, 10_000])
def test_host_loop_schedule(pkg, tmp_path, hdf5_step):
    """Groups before steps 0, k, 2k, ... (k = hdf5_step) while steps remain;
    FILE_NUM = groups + 1; grid and initial particle coordinates, nid and the
    BC arrays at the root."""
    c = pkg.workloads.column_collapse_2d(h=0.02, Ttol=0.01, hdf5=True, hdf5_step=hdf5_step,
                                         project_path=str(tmp_path))
    nsteps = pkg.time_sequence(c.args)
    dev = _FakeDevice(c.mp)
    pkg.solver._run_with_snapshots(c.args, c.grid, c.mp, c.attr, c.bc, dev, nsteps, None)
    expect = list(range(0, nsteps, hdf5_step))
    assert [s for _, s, _ in dev.calls] == expect
    assert [g for g, _, _ in dev.calls] == list(range(1, len(expect) + 1))
    t = pkg.hdf5.read(pkg.snapshot_path(c.args))
    assert t["FILE_NUM"] == len(expect) + 1
    assert np.array_equal(t["grid_coords"].T, c.grid.xi)
    assert np.array_equal(t["mp_coords0"].T, c.mp.xi0)
    assert np.array_equal(t["nid"], c.attr.nid)
    for a in ("x", "y"):
        assert np.array_equal(t[f"vbc_{a}s_idx"], getattr(c.bc, f"v{a}_s_idx"))
        assert np.array_equal(t[f"vbc_{a}s_val"], getattr(c.bc, f"v{a}_s_val"))
    # time of group i = the loop's Ti before step (i-1)*k, accumulated in T2
    Ti, k = 0.0, 0
    for g, s, T in dev.calls:
        while k < s:
            Ti = float(np.float64(Ti) + np.float64(c.args.dT))
            k += 1
        assert t[f"group{g}"]["time"] == Ti


def test_snapshot_mask_constant(pkg):
    import re
    hdr = open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                            "include", "mpm_b200.h")).read()
    m = re.search(r"#define MPM_F_SNAPSHOT \((.*?)\)\n", hdr, flags=re.S)
    names = re.findall(r"MPM_F_(\w+)", m.group(1))
    L = pkg._lib
    assert sum(getattr(L, "F_" + n) for n in names) == L.F_SNAPSHOT


# ---- GPU -------------------------------------------------------------------------

FIELDS = {"stress": "sig", "strain_s": "eps", "eqstrain": "epsq", "ekstrain": "epsk", "eqrate": "epsv",
          "coords": "xi", "velocity_s": "vs", "volume": "Omega", "mass_s": "ms"}


@pytest.mark.gpu
@pytest.mark.parametrize("precision,gpu_precision", [("FP64", "fp64"), ("FP64", "mixed"), ("FP32", "mixed")])
def test_snapshots_equal_downloads(pkg, gpu_lib, tmp_path, precision, gpu_precision):
    """Each group holds exactly what a download of the same device state
    returns (the snapshot is taken, then the download, then the next steps)."""
    k = 40
    c = pkg.workloads.column_collapse_2d(h=0.01, Ttol=0.02, precision=precision, gpu_precision=gpu_precision)
    T = np.float32 if precision == "FP32" else np.float64
    dev = pkg.DeviceModel(c.args, c.grid, c.mp, c.attr, c.bc)
    f = pkg.hdf5.H5File(tmp_path / "s.h5")
    refs = []
    try:
        Ti = T(0.0)
        for g in range(1, 5):
            dev.snapshot(f, g, float(Ti), dtype=T)
            out = fresh_particles(pkg, c.mp)
            dev.download(pkg._lib.F_SNAPSHOT, out)
            refs.append((Ti, out))
            Ti = T(dev.step(c.dt, float(Ti), k))
        assert dev.snapshot_wait() == 4
    finally:
        dev.close()
        f.close()
    t = pkg.hdf5.read(tmp_path / "s.h5")
    for g, (Ti, out) in enumerate(refs, start=1):
        grp = t[f"group{g}"]
        assert grp["time"] == Ti and grp["time"].dtype == T
        for name, attr in FIELDS.items():
            got = grp[name]
            assert got.dtype == T, name
            assert np.array_equal(got.T if got.ndim == 2 else got, getattr(out, attr)), (g, name)


@pytest.mark.gpu
@pytest.mark.parametrize("precision,gpu_precision,tol", [("FP64", "fp64", 1e-9), ("FP32", "mixed", 1e-4)])
def test_solver_hdf5_run(pkg, gpu_lib, tmp_path, precision, gpu_precision, tol):
    """materialpointsolver with hdf5 = true: one group per hdf5_step steps,
    matching a second model stepped by the same chunks (to the run-to-run
    spread of the floating-point reductions), and the final state downloaded."""
    k = 40
    kw = dict(h=0.01, Ttol=0.02, precision=precision, gpu_precision=gpu_precision, hdf5=True, hdf5_step=k)
    c = pkg.workloads.column_collapse_2d(project_path=str(tmp_path), **kw)
    pkg.materialpointsolver(c.args, c.grid, c.mp, c.attr, c.bc)
    t = pkg.hdf5.read(pkg.snapshot_path(c.args))
    nsteps = pkg.time_sequence(c.args)
    ngroups = len(range(0, nsteps, k))
    assert ngroups >= 3 and t["FILE_NUM"] == ngroups + 1
    c2 = pkg.workloads.column_collapse_2d(project_path=str(tmp_path / "ref"), **dict(kw, hdf5=False))
    dev = pkg.DeviceModel(c2.args, c2.grid, c2.mp, c2.attr, c2.bc)
    T = np.float32 if precision == "FP32" else np.float64
    try:
        Ti, done = T(0.0), 0
        for g in range(1, ngroups + 1):
            out = fresh_particles(pkg, c2.mp)
            dev.download(pkg._lib.F_SNAPSHOT, out)
            grp = t[f"group{g}"]
            assert grp["time"] == Ti and grp["time"].dtype == T
            for name in ("coords", "velocity_s", "stress", "volume"):
                got = grp[name]
                got = got.T if got.ndim == 2 else got
                ref = getattr(out, FIELDS[name])
                if name == "coords":   # compare displacements, not positions
                    got, ref = got - c2.mp.xi0, ref - c2.mp.xi0
                assert rel(got, ref) <= tol, (g, name, rel(got, ref))
            n = min(k, nsteps - done)
            Ti = T(dev.step(c2.dt, float(Ti), n))
            done += n
        out = fresh_particles(pkg, c2.mp)
        dev.download(pkg._lib.F_REFERENCE, out)
        assert rel(c.mp.xi - c.mp.xi0, out.xi - c2.mp.xi0) <= tol
    finally:
        dev.close()


@pytest.mark.gpu
def test_snapshot_is_asynchronous_and_rejects_bad_masks(pkg, gpu_lib, tmp_path):
    c = pkg.workloads.column_collapse_2d(h=0.01, Ttol=0.01)
    dev = pkg.DeviceModel(c.args, c.grid, c.mp, c.attr, c.bc)
    f = pkg.hdf5.H5File(tmp_path / "s.h5")
    try:
        with pytest.raises(pkg._lib.MPMError, match="MPM_F_SNAPSHOT"):
            dev.snapshot(f, 1, 0.0, fields=pkg._lib.F_F)
        Ti = 0.0
        for g in range(1, 6):            # more snapshots than slots: the third waits for the first
            dev.snapshot(f, g, Ti, fields=pkg._lib.F_XI | pkg._lib.F_SIG)
            Ti = dev.step(c.dt, Ti, 5)
        assert dev.snapshot_wait() == 5
    finally:
        dev.close()
        f.close()
    t = pkg.hdf5.read(tmp_path / "s.h5")
    assert sorted(t) == [f"group{g}" for g in range(1, 6)]
    assert set(t["group3"]) == {"coords", "stress", "time"}
