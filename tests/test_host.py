"""Host-side types and helpers (CPU): argument validation as in
src/types/modelargs.jl, node ordering as in src/types/grid.jl, the time loop
of submit_work! (src/solver.jl), the workloads' sizes, the descriptor the
binding sends to the library."""
import math

import numpy as np
import pytest


def _args(pkg, tmp_path, dim=3, **kw):
    base = dict(Ttol=0.1, dT=1e-4, constitutive="linearelastic", project_name="t",
                project_path=str(tmp_path), device="B200")
    base.update(kw)
    return (pkg.types.Args3D if dim == 3 else pkg.types.Args2D)(**base)


@pytest.mark.parametrize("kw,msg", [
    (dict(Ttol=0.0), "Simulation time"),
    (dict(dT=1.0), "Time step cannot"),
    (dict(Te=1.0), "Elastic loading"),
    (dict(basis="cubic"), "basis"),
    (dict(FLIP=0.5), r"FLIP\+PIC"),
    (dict(zeta_s=2.0), "ζs"),
    (dict(project_name=""), "Empty project"),
    (dict(coupling="XX"), "Coupling"),
    (dict(device="TPU"), "device"),
    (dict(va="b"), "velocity update"),
])
def test_args_validation(pkg, tmp_path, kw, msg):
    with pytest.raises(ValueError, match=msg):
        _args(pkg, tmp_path, **kw)


def test_args_unicode_aliases(pkg, tmp_path):
    a = _args(pkg, tmp_path, **{"ζs": 0.05})
    assert a.zeta_s == 0.05


def test_grid2d_node_order(pkg):
    """2D nodes: columns along x, y DESCENDING inside a column (grid.jl:92-100)."""
    g = pkg.types.Grid2D(x1=0.0, x2=0.3, y1=0.0, y2=0.2, dx=0.1, dy=0.1)
    assert (g.nnx, g.nny, g.ni, g.nc) == (4, 3, 12, 6)
    assert np.allclose(g.xi[:3], [[0, 0.2], [0, 0.1], [0, 0.0]])
    assert np.allclose(g.xi[3], [0.1, 0.2])


def test_grid3d_node_order(pkg):
    """3D nodes: y fastest, then x, then z (grid.jl:236-249)."""
    g = pkg.types.Grid3D(x1=0.0, x2=0.2, y1=0.0, y2=0.3, z1=0.0, z2=0.1, dx=0.1, dy=0.1, dz=0.1)
    assert (g.nnx, g.nny, g.nnz) == (3, 4, 2)
    xi = g.xi
    assert np.allclose(xi[1], [0, 0.1, 0]) and np.allclose(xi[4], [0.1, 0, 0])
    assert np.allclose(xi[12], [0, 0, 0.1])


def test_grid_validation(pkg):
    with pytest.raises(ValueError):
        pkg.types.Grid2D(x1=1.0, x2=0.0, y1=0.0, y2=1.0, dx=0.1, dy=0.1)
    with pytest.raises(ValueError):
        pkg.types.Grid3D(x1=0.0, x2=1.0, y1=0.0, y2=1.0, z1=0.0, z2=1.0, dx=0.1, dy=-0.1, dz=0.1)


def test_time_sequence_matches_julia_loop(pkg, tmp_path):
    """`while Ti < Ttol; …; Ti += ΔT` in the model's float type."""
    # ten additions of 0.1 give 0.9999999999999999 < 1.0: the loop runs 11 times
    a = _args(pkg, tmp_path, Ttol=1.0, dT=0.1)
    Ti, k = 0.0, 0
    while Ti < 1.0:
        Ti += 0.1
        k += 1
    assert pkg.solver.time_sequence(a) == k == 11
    a32 = _args(pkg, tmp_path, Ttol=0.3, dT=0.1, precision="FP32")
    Ti, k = np.float32(0), 0
    while Ti < np.float32(0.3):
        Ti = np.float32(Ti + np.float32(0.1))
        k += 1
    assert pkg.solver.time_sequence(a32) == k


def test_workload_sizes(pkg):
    c2 = pkg.workloads.column_collapse_2d()
    assert c2.mp.np == 3200 and c2.grid.dim == 2
    assert c2.args.constitutive == "druckerprager"
    c3 = pkg.workloads.column_collapse_3d(h=0.02)
    # the column (0.5 x 0.2 x 0.4 m) at 2 particles per cell and axis
    assert c3.mp.np == 25 * 10 * 20 * 8


def test_make_desc(pkg):
    c = pkg.workloads.column_collapse_3d(h=0.04, column=(0.08, 0.08, 0.08), domain=(0.16, 0.12, 0.12))
    d = pkg.solver.make_desc(c.args, c.grid, c.mp, c.attr)
    assert d.dim == 3 and d.np == c.mp.np and d.abi_version == pkg._lib.ABI_VERSION
    assert (d.nnx, d.nny, d.nnz) == (c.grid.nnx, c.grid.nny, c.grid.nnz)
    assert (d.dx, d.lpx) == (c.grid.dx, c.mp.dx)
    assert d.constitutive == pkg._lib.MOHRCOULOMB and d.mc3d == 0
    assert d.gravity == c.args.gravity and d.FLIP == c.args.FLIP


def test_host_views_layout(pkg):
    """Views point at the host arrays themselves, column-major with ld = np."""
    c = pkg.workloads.column_collapse_2d(h=0.02)
    v = pkg.solver.host_views(c.grid, c.mp, c.attr, c.bc)
    assert v.xi.ptr == c.mp.xi.ctypes.data and v.xi.ld == c.mp.np
    assert v.xi.type == pkg._lib.T_F64
    assert v.nid.type == pkg._lib.T_I64
    assert v.vz_idx.ptr is None


def test_entry_point_rejects_other_devices(pkg, tmp_path):
    c = pkg.workloads.column_collapse_2d(h=0.02)
    c.args.device = "CUDA"
    with pytest.raises(ValueError):
        pkg.materialpointsolver(c.args, c.grid, c.mp, c.attr, c.bc)
