"""GPU parity: the sm_100a library through its C ABI against the FP64 oracle.

Tolerances (relative, norm-wise over all particles): the all-FP64 device mode
must agree with the oracle to 1e-9 (only the summation order of atomics
differs).  The mixed mode (FP32 bulk, FP64 positions and det F) must agree to
1e-4 in displacement, velocity, F and volume, and to 1e-3 in stress and strain:
near the free surface the strain signal is ~1e-3 of the rigid-motion part of
the nodal displacement increments, which FP32 nodal storage resolves only to
~1e-5 relative per step.  p2c and the cell sort are compared bit-exactly.
"""
import numpy as np
import pytest

from helpers import fresh_particles, rel

pytestmark = pytest.mark.gpu

TOL64 = 1e-9
TOL32 = 1e-4
TOL32_STRESS = 1e-3


def tol_stress(tol):
    return TOL32_STRESS if tol == TOL32 else tol


def run_both(pkg, orc, case, nsteps, tiled=False, box=True, variant=None):
    import os
    lib = pkg._lib
    env = {"MPM_B200_TILED": "1" if tiled else "0", "MPM_B200_BOX": "1" if box else "0"}
    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        dev = pkg.DeviceModel(case.args, case.grid, case.mp, case.attr, case.bc)
    finally:
        for k, v in old.items():
            if v is None:
                del os.environ[k]
            else:
                os.environ[k] = v
    if variant is not None:
        dev.set_tuning(dev.tuning()[0], variant)
    dev.step(case.dt, 0.0, nsteps)
    out = fresh_particles(pkg, case.mp)
    dev.download(lib.F_REFERENCE | lib.F_F, out)
    dev.close()
    o = orc.Oracle(case.args, case.grid, case.mp, case.attr, case.bc)
    o.run(case.dt, 0.0, nsteps)
    return out, o


def check_fields(out, o, mp0, tol, tol_s=None):
    tol_s = tol if tol_s is None else tol_s
    du_g = out.xi - mp0.xi
    du_o = o.xi - mp0.xi
    assert rel(du_g, du_o) < tol, ("displacement", rel(du_g, du_o))
    assert rel(out.vs, o.vs) < tol, ("velocity", rel(out.vs, o.vs))
    assert rel(out.F, o.F) < tol, ("F", rel(out.F, o.F))
    assert rel(out.Omega, o.Omega) < tol, ("volume", rel(out.Omega, o.Omega))
    assert rel(out.sig, o.sig) < tol_s, ("stress", rel(out.sig, o.sig))
    assert rel(out.eps, o.eps) < tol_s, ("strain", rel(out.eps, o.eps))
    assert rel(out.sigm, o.sigm) < tol_s, ("sigm", rel(out.sigm, o.sigm))
    assert rel(out.epsv, o.epsv) < tol_s * 10, ("strain rate", rel(out.epsv, o.epsv))
    if np.abs(o.epsq).max() > 0:
        assert rel(out.epsq, o.epsq) < tol_s * 10, ("epsq", rel(out.epsq, o.epsq))


def small2d(pkg, **kw):
    base = dict(h=0.01, width=0.1, height=0.06, domain=(0.2, 0.1), seed=11)
    base.update(kw)
    return pkg.workloads.column_collapse_2d(**base)


def small3d(pkg, **kw):
    base = dict(h=0.02, column=(0.12, 0.08, 0.12), domain=(0.24, 0.12, 0.16), seed=12)
    base.update(kw)
    return pkg.workloads.column_collapse_3d(**base)


@pytest.mark.parametrize("prec,tol", [("fp64", TOL64), ("mixed", TOL32)])
@pytest.mark.parametrize("model", ["linearelastic", "druckerprager", "mohrcoulomb"])
def test_steps_2d(pkg, orc, gpu_lib, prec, tol, model):
    case = small2d(pkg, constitutive=model, gpu_precision=prec)
    out, o = run_both(pkg, orc, case, 12)
    check_fields(out, o, case.mp, tol, tol_stress(tol))


@pytest.mark.parametrize("prec,tol", [("fp64", TOL64), ("mixed", TOL32)])
@pytest.mark.parametrize("model", ["linearelastic", "druckerprager", "mohrcoulomb"])
def test_steps_3d(pkg, orc, gpu_lib, prec, tol, model):
    case = small3d(pkg, constitutive=model, gpu_precision=prec)
    out, o = run_both(pkg, orc, case, 8)
    check_fields(out, o, case.mp, tol, tol_stress(tol))


def mc3d_case(pkg, prec):
    """Cohesive Mohr-Coulomb column (c = 500 Pa, σt = 200 Pa) with a seeded
    compressive prestress near the yield surface, so that almost every particle
    yields in the first steps, away from the cone apex.  (For c = 0 and σt = 0
    the restated return is singular at the apex, ρ -> 0 with a zero-offset
    tension potential: particles at the free surface then get arbitrary plastic
    multipliers in the oracle as well, so that case carries no parity.)"""
    case = small3d(pkg, constitutive="mohrcoulomb", mc3d="restated", gpu_precision=prec, c=500.0, sigt=200.0)
    rng = np.random.default_rng(77)
    n = case.mp.np
    case.mp.sig[:, :3] = rng.normal(-4000.0, 1500.0, (n, 3))
    case.mp.sig[:, 3:] = rng.normal(0.0, 1000.0, (n, 3))
    return case


# The restated return is discontinuous at the yield surface: its first
# corrector takes the multiplier from the pre-increment stress when that stress
# is within 0.1 Pa of the surface, else from the trial stress, and the two land
# on different points of the surface.  A returned stress stored in FP32 (as the
# mixed mode stores every particle stress) moves by ~1e-4 Pa and flips that
# choice for a fraction of the yielding particles on their next step.  The
# oracle itself shows it: rounding its stresses to FP32 after every step moves
# its 20-step result by 4e-3 in displacement and 8e-2 in stress.  The mixed
# mode is held to twice that self-difference of the oracle, field by field;
# the FP64 mode shows the device return itself is exact.
MC3D_FIELDS = ("vs", "sig", "eps", "F", "Omega", "sigm", "epsv", "epsq")


def oracle_fp32_stress_spread(pkg, orc, case_fn, nsteps):
    """Per-field relative difference between the FP64 oracle and the same
    oracle with its particle stresses rounded to FP32 after every step."""
    a, b = case_fn(), case_fn()
    oa = orc.Oracle(a.args, a.grid, a.mp, a.attr, a.bc)
    oa.run(a.dt, 0.0, nsteps)
    ob = orc.Oracle(b.args, b.grid, b.mp, b.attr, b.bc)
    ob.sig[:] = ob.sig.astype(np.float32)
    Ti = 0.0
    for _ in range(nsteps):
        ob.procedure(b.dt, Ti)
        Ti += b.dt
        ob.sig[:] = ob.sig.astype(np.float32)
    spread = {f: rel(getattr(ob, f), getattr(oa, f)) for f in MC3D_FIELDS}
    spread["disp"] = rel(ob.xi - b.mp.xi, oa.xi - a.mp.xi)
    return spread


@pytest.mark.parametrize("tiled", [False, True])
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_mc3d_restated(pkg, orc, gpu_lib, prec, tiled):
    """The restated 3D Mohr-Coulomb return (FP64 on the device in both modes)
    against the oracle's restatement, over steps where almost all particles
    yield."""
    nsteps = 20
    case = mc3d_case(pkg, prec)
    out, o = run_both(pkg, orc, case, nsteps, tiled=tiled)
    assert (o.epsq > 0).mean() > 0.9
    if prec == "fp64":
        check_fields(out, o, case.mp, TOL64)
        return
    spread = oracle_fp32_stress_spread(pkg, orc, lambda: mc3d_case(pkg, "fp64"), nsteps)
    got = {f: rel(getattr(out, f), getattr(o, f)) for f in MC3D_FIELDS}
    got["disp"] = rel(out.xi - case.mp.xi, o.xi - case.mp.xi)
    for f, err in got.items():
        bound = max(TOL32, 2.0 * spread[f])
        assert err < bound, (f, err, bound, spread[f])


@pytest.mark.parametrize("prec,tol", [("fp64", TOL64), ("mixed", TOL32)])
@pytest.mark.parametrize("dim", [2, 3])
def test_tiled_path(pkg, orc, gpu_lib, dim, prec, tol):
    """The shared-memory tiled particle passes compute the same step."""
    mk = small2d if dim == 2 else small3d
    case = mk(pkg, constitutive="druckerprager", gpu_precision=prec)
    out, o = run_both(pkg, orc, case, 8, tiled=True)
    check_fields(out, o, case.mp, tol, tol_stress(tol))


@pytest.mark.parametrize("variant", [0, 2, 3])
@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("model", ["linearelastic", "druckerprager"])
def test_box_and_chain_passes(pkg, orc, gpu_lib, dim, model, variant):
    """The mixed-mode step through the per-particle lane-merged passes (variant
    0; 3: the fused pass compiled for 3 resident CTAs per SM) and through the
    shared-memory box passes (2: one warp per tile), each against the oracle."""
    mk = small2d if dim == 2 else small3d
    case = mk(pkg, constitutive=model, gpu_precision="mixed", sort_every=8)
    out, o = run_both(pkg, orc, case, 24, box=variant == 2, variant=variant)
    check_fields(out, o, case.mp, TOL32, TOL32_STRESS)


@pytest.mark.parametrize("tiled", [False, True])
@pytest.mark.parametrize("prec,tol", [("fp64", TOL64), ("mixed", 1e-3)])
def test_drift_beyond_tile_margin(pkg, orc, gpu_lib, prec, tol, tiled):
    """No re-sort for 120 steps while the column translates by > 2 cells: the
    particles leaving their tile's window (tiled passes) or their tile's node
    box (box passes, the mixed-mode default) take the global path.  Mixed mode is
    checked on the kinematics only: the elastic velocities (~1e-3 m/s) ride on
    a 3 m/s translation, and FP32 nodal velocities resolve them to ~1e-3, so
    the stresses they integrate differ from FP64 by up to ~10 % -- the same
    limit the reference has in its FP32 mode."""
    case = small3d(pkg, constitutive="linearelastic", gpu_precision=prec, sort_every=100000,
                   domain=(0.4, 0.12, 0.16))
    case.mp.xi[:, 0] += 0.05          # away from the fixed wall
    case.mp.vs[:, 0] = 3.0
    out, o = run_both(pkg, orc, case, 120, tiled=tiled)
    moved = np.abs(o.xi[:, 0] - case.mp.xi[:, 0]).max() / case.grid.dx
    assert moved > 2.0
    if prec == "fp64":
        check_fields(out, o, case.mp, tol)
    else:
        assert rel(out.xi - case.mp.xi, o.xi - case.mp.xi) < tol
        assert rel(out.vs, o.vs) < tol


@pytest.mark.parametrize("dim", [2, 3])
def test_va_v_and_pic(pkg, orc, gpu_lib, dim):
    mk = small2d if dim == 2 else small3d
    case = mk(pkg, constitutive="druckerprager", gpu_precision="fp64", va="v", FLIP=0.7, PIC=0.3)
    out, o = run_both(pkg, orc, case, 6)
    check_fields(out, o, case.mp, TOL64)


def test_bc_values(pkg, orc, gpu_lib):
    case = small2d(pkg, constitutive="druckerprager", gpu_precision="fp64")
    # a moving left wall: non-zero prescribed x velocity (the as <- val quirk of
    # solvegrid_a_OS!, utils_OS.jl:575-578, is exercised too)
    vals = np.where(case.bc.vx_s_idx != 0, 0.01, 0.0)
    case.bc.vx_s_val[:] = vals
    out, o = run_both(pkg, orc, case, 6)
    check_fields(out, o, case.mp, TOL64)


def test_damping(pkg, orc, gpu_lib):
    """Local damping -ζs·|f|·sign(vs) (utils_OS.jl:563-567) is discontinuous in
    vs at 0: nodal velocities that are zero up to rounding take their sign from
    the summation order of the atomics, so agreement is to 1e-4, not 1e-9."""
    case = small2d(pkg, constitutive="druckerprager", gpu_precision="fp64", ζs=0.05)
    out, o = run_both(pkg, orc, case, 6)
    check_fields(out, o, case.mp, 1e-4)


def test_gravity_ramp(pkg, orc, gpu_lib):
    case = small2d(pkg, constitutive="druckerprager", gpu_precision="fp64", Te=0.5 * 1e-3, Ttol=1.0)
    out, o = run_both(pkg, orc, case, 20)
    check_fields(out, o, case.mp, TOL64)


def test_ramp_in_chunks(pkg, orc, gpu_lib):
    """The P2G a fused pass leaves behind is reused by the next mpm_step call
    when the caller's Ti gives the same gravity, and redone when it does not
    (inside the ramp Ti < Te every Ti has its own gravity).  Chunked calls
    across the ramp match the oracle's single run, and the standalone P2G runs
    exactly where the rule says."""
    Te = 0.5 * 1e-3
    case = small2d(pkg, constitutive="druckerprager", gpu_precision="fp64", Te=Te, Ttol=1.0)

    def stepper(dev):
        runs = [0]

        def step(Ti, n):
            Ti = dev.step(case.dt, Ti, n)
            kt = dev.kernel_times()
            runs[0] += kt.get("p2g", (0.0, 0))[1]
            assert kt["g2p_p2g"][1] == n
            return Ti
        return step, runs

    dev = pkg.DeviceModel(case.args, case.grid, case.mp, case.attr, case.bc)
    try:
        dev.set_profiling(True)
        step, runs = stepper(dev)
        Ti = step(0.0, 5)
        assert runs[0] == 1
        for _ in range(3):                      # continuing at the returned Ti
            Ti = step(Ti, 5)
        assert runs[0] == 1 and Ti > Te
        out = fresh_particles(pkg, case.mp)
        dev.download(pkg._lib.F_REFERENCE | pkg._lib.F_F, out)
        step(Ti * (1 + 1e-12), 2)               # past the ramp: same gravity, reused
        assert runs[0] == 1
    finally:
        dev.close()
    o = orc.Oracle(case.args, case.grid, case.mp, case.attr, case.bc)
    o.run(case.dt, 0.0, 20)
    check_fields(out, o, case.mp, TOL64)
    dev = pkg.DeviceModel(case.args, case.grid, case.mp, case.attr, case.bc)
    try:
        dev.set_profiling(True)
        step, runs = stepper(dev)
        Ti = step(0.0, 3)
        step(Ti * (1 + 1e-12), 3)               # inside the ramp: another gravity, redone
        assert runs[0] == 2
    finally:
        dev.close()


@pytest.mark.parametrize("dim", [2, 3])
def test_p2g_stage(pkg, orc, gpu_lib, dim):
    mk = small2d if dim == 2 else small3d
    case = mk(pkg, constitutive="linearelastic", gpu_precision="fp64")
    # give the particles stress and velocity so every P2G term is exercised
    rng = np.random.default_rng(5)
    case.mp.sig[:] = rng.normal(0, 1e3, case.mp.sig.shape)
    case.mp.vs[:] = rng.normal(0, 0.1, case.mp.vs.shape)
    dev = pkg.DeviceModel(case.args, case.grid, case.mp, case.attr, case.bc)
    dev.run_stages(case.dt, 0.0, 1)
    m_g = dev.grid_field(0)
    p_g = dev.grid_field(1)
    f_g = dev.grid_field(2)
    dev.close()
    o = orc.Oracle(case.args, case.grid, case.mp, case.attr, case.bc)
    o.stage("resetgrid")
    o.stage("resetmp")
    o.stage("p2g", case.args.gravity)
    assert rel(m_g, o.g_ms) < 1e-12
    assert rel(p_g, o.g_ps) < 1e-12
    assert rel(f_g, o.g_fs) < 1e-12


@pytest.mark.parametrize("user_precision,cut", [("FP64", False), ("FP32", True)])
@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_massless_cutoff_follows_reference_precision(pkg, gpu_lib, prec, user_precision, cut):
    """The solve treats a node as massless when m < eps(T2), T2 the reference's
    float type (utils_OS.jl:515, 555): with FP64 inputs a node of ~1e-9 kg moves
    with its momentum, with FP32 inputs it is cut (velocity 0) -- whatever the
    device stores.  (Cutting at FP32's eps in the mixed mode of an FP64 problem
    froze the light boundary nodes of the reference's 3D validation column,
    2.5 mm cells, and the USL run blew up.)"""
    case = small2d(pkg, constitutive="linearelastic", gpu_precision=prec, precision=user_precision, rho=1e-4,
                   gravity=0.0)
    case.mp.vs[:, 0] = 1.0
    dev = pkg.DeviceModel(case.args, case.grid, case.mp, case.attr, case.bc)
    try:
        dev.run_stages(case.dt, 0.0, 1 | 2)          # P2G, solve
        m = dev.grid_field(0)
        vT = dev.grid_field(3)
    finally:
        dev.close()
    free = (m > 0) & (case.bc.vx_s_idx == 0) & (case.bc.vy_s_idx == 0)
    assert free.sum() > 20
    assert m[free].max() < 1e-7 and m[free].min() > 1e-15
    if cut:
        assert not vT[free].any()
    else:
        assert np.allclose(vT[free, 0], 1.0, rtol=1e-5) and np.allclose(vT[free, 1], 0.0, atol=1e-6)


@pytest.mark.parametrize("dim", [2, 3])
def test_p2c_bit_exact(pkg, orc, gpu_lib, dim):
    mk = small2d if dim == 2 else small3d
    case = mk(pkg)
    g = case.grid
    rng = np.random.default_rng(7)
    xi = case.mp.xi.copy(order="F")
    n = xi.shape[0]
    # a quarter of the particles exactly on node lines (the fld/cld rule decides)
    k = n // 4
    for d, (a1, h, nn) in enumerate([(g.x1, g.dx, g.nnx), (g.y1, g.dy, g.nny)] +
                                    ([(g.z1, g.dz, g.nnz)] if dim == 3 else [])):
        j = rng.integers(3, nn - 3, size=k)
        xi[:k, d] = a1 + j * h
    case.mp.xi[:] = xi
    dev = pkg.DeviceModel(case.args, case.grid, case.mp, case.attr, case.bc)
    p_gpu = dev.p2c()
    dev.close()
    o = orc.Oracle(case.args, case.grid, case.mp, case.attr, case.bc)
    p_ref = o.p2c(case.mp.xi)
    assert np.array_equal(p_gpu, p_ref)


TILE = {3: (2, 8, 2), 2: (4, 8, 1)}   # the library's default sort tiles (32 cells)


def host_cells(p2c, g, dim):
    q = p2c - 1
    cy = q % g.ncy
    cx = (q // g.ncy) % g.ncx
    cz = q // (g.ncy * g.ncx) if dim == 3 else np.zeros_like(q)
    return cx, cy, cz


def host_key(p2c, g, dim):
    """Tile-major cell key (the default tiles) from the 1-based p2c."""
    cx, cy, cz = host_cells(p2c, g, dim)
    TX, TY, TZ = TILE[dim]
    ntx = -(-g.ncx // TX)
    nty = -(-g.ncy // TY)
    tx, ty, tz = cx // TX, cy // TY, cz // TZ
    lx, ly, lz = cx - tx * TX, cy - ty * TY, cz - tz * TZ
    t = (tz * ntx + tx) * nty + ty
    return t * (TX * TY * TZ) + (lz * TX + lx) * TY + ly


def host_octant(xi, p2c, g, dim):
    """Sub-cell octant: bit a set when the offset from the cell's first node is
    at least half a cell (the same FP64 operations as the device)."""
    cells = host_cells(p2c, g, dim)
    x1 = (g.x1, g.y1, g.z1 if dim == 3 else 0.0)
    h = (g.dx, g.dy, g.dz if dim == 3 else 1.0)
    o = np.zeros(len(p2c), np.int64)
    for a in range(dim):
        s = xi[:, a] - (x1[a] + cells[a].astype(np.float64) * h[a])
        o |= (s >= 0.5 * h[a]).astype(np.int64) << a
    return o


@pytest.mark.parametrize("dim", [2, 3])
def test_sort_bit_exact(pkg, orc, gpu_lib, dim):
    mk = small2d if dim == 2 else small3d
    case = mk(pkg)
    rng = np.random.default_rng(3)
    perm = rng.permutation(case.mp.np)
    for name in ("xi",):
        getattr(case.mp, name)[:] = getattr(case.mp, name)[perm]
    dev = pkg.DeviceModel(case.args, case.grid, case.mp, case.attr, case.bc)
    dev.sort()
    order = dev.order()
    dev.close()
    o = orc.Oracle(case.args, case.grid, case.mp, case.attr, case.bc)
    p2c = o.p2c(case.mp.xi)
    key = host_key(p2c, case.grid, dim)
    octant = host_octant(case.mp.xi, p2c, case.grid, dim)
    cpt = 32
    # rank of each particle within its cell, by (octant, original index)
    by_cell = np.lexsort((np.arange(case.mp.np), octant, key))
    rank = np.empty(case.mp.np, np.int64)
    ks = key[by_cell]
    start = np.r_[0, np.flatnonzero(np.diff(ks)) + 1]
    lens = np.diff(np.r_[start, len(ks)])
    rank[by_cell] = np.arange(len(ks)) - np.repeat(start, lens)
    expect = np.lexsort((key % cpt, rank, key // cpt))
    assert np.array_equal(order, expect)


def test_out_of_grid_reported(pkg, gpu_lib):
    case = small2d(pkg)
    case.mp.xi[0, 0] = case.grid.x1 + 0.2 * case.grid.dx   # inside the first cell: stencil leaves the grid
    dev = pkg.DeviceModel(case.args, case.grid, case.mp, case.attr, case.bc)
    with pytest.raises(pkg._lib.MPMError) as ei:
        dev.step(case.dt, 0.0, 1)
    assert ei.value.code == -3
    dev.close()


def test_nan_reported(pkg, gpu_lib):
    case = small2d(pkg, constitutive="linearelastic")
    case.mp.sig[3, 0] = np.nan
    dev = pkg.DeviceModel(case.args, case.grid, case.mp, case.attr, case.bc)
    with pytest.raises(pkg._lib.MPMError) as ei:
        dev.step(case.dt, 0.0, 2)
    assert ei.value.code == -5
    dev.close()


def test_entry_point_matches_oracle(pkg, orc, gpu_lib):
    """materialpointsolver(...) end to end (upload, loop, device2host!, free)."""
    case = small2d(pkg, constitutive="druckerprager", gpu_precision="fp64", Ttol=40 * 2.2e-4)
    import copy
    mp0 = copy.deepcopy(case.mp)
    pkg.materialpointsolver(case.args, case.grid, case.mp, case.attr, case.bc)
    n = pkg.time_sequence(case.args)
    o = orc.Oracle(case.args, case.grid, mp0, case.attr, case.bc)
    o.run(case.args.dT, 0.0, n)
    assert rel(case.mp.xi - mp0.xi, o.xi - mp0.xi) < TOL64
    assert rel(case.mp.sig, o.sig) < TOL64
    assert rel(case.mp.ms, o.ms) < 1e-12


@pytest.mark.parametrize("prec,tol", [("fp64", TOL64), ("mixed", TOL32)])
def test_slope_random_cohesion(pkg, orc, gpu_lib, prec, tol):
    """3D slope with one material per particle whose cohesion is a lognormal
    random field (the reference's nid = 1:np form).  The library stores it as
    one material record plus a per-particle cohesion that travels through the
    cell sort; the oracle keeps the 3 184 material records."""
    case = pkg.workloads.slope_3d(h=0.5, domain=(20.0, 4.0, 10.0), height=3.0, crest=2.0, corr_len=1.0, nh=500,
                                  Te=0.0, gpu_precision=prec, seed=31, sort_every=4, c_mean=1.0e3)
    assert len(case.attr.c) == case.mp.np and np.ptp(case.attr.c) > 0
    out, o = run_both(pkg, orc, case, 20)
    assert (o.epsq > 1e-9).mean() > 0.2
    check_fields(out, o, case.mp, tol, tol_stress(tol))


@pytest.mark.parametrize("dim", [2, 3])
def test_graph_replay_matches_direct_launches(pkg, orc, gpu_lib, dim, monkeypatch):
    """Steps after the gravity ramp are replayed from captured CUDA graphs in
    blocks of two sort periods; the same 40 steps issued launch by launch give
    the same state (FP64 mode: only the order of atomic additions differs), and
    both match the oracle."""
    mk = small2d if dim == 2 else small3d
    outs, stats = [], []
    for graphs in ("1", "0"):
        monkeypatch.setenv("MPM_B200_GRAPHS", graphs)
        case = mk(pkg, constitutive="druckerprager", gpu_precision="fp64")
        dev = pkg.DeviceModel(case.args, case.grid, case.mp, case.attr, case.bc)
        dev.step(case.dt, 0.0, 40)
        out = fresh_particles(pkg, case.mp)
        dev.download(pkg._lib.F_REFERENCE | pkg._lib.F_F, out)
        stats.append(dev.stats())
        dev.close()
        outs.append(out)
    assert stats[0].steps_done == stats[1].steps_done == 40
    assert stats[0].sorts_done == stats[1].sorts_done
    assert stats[0].launches == stats[1].launches
    for f in ("xi", "vs", "sig", "F"):
        assert rel(getattr(outs[0], f), getattr(outs[1], f)) < 1e-12, f
    o = orc.Oracle(case.args, case.grid, case.mp, case.attr, case.bc)
    o.run(case.dt, 0.0, 40)
    check_fields(outs[0], o, case.mp, TOL64)


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
@pytest.mark.parametrize("mvl", [False, True])
@pytest.mark.parametrize("scheme", ["MUSL", "USL"])
@pytest.mark.parametrize("dim", [2, 3])
def test_lane_merged_scatter_matches_plain(pkg, orc, gpu_lib, dim, scheme, mvl, prec, monkeypatch):
    """The particle passes merge the scatters of warp lanes whose windows
    are consecutive in y (k_g2p_chain / k_dmap_chain, and k_mvl_p2g_chain with
    MVL); with the merging off (MPM_B200_CHAIN=0) the plain per-lane
    reductions run.  Both are the same sums in another order: they agree to
    rounding (FP32 or FP64), and both match the oracle to that mode's tolerance."""
    mk = small2d if dim == 2 else small3d
    outs = []
    for chain in ("1", "0"):
        monkeypatch.setenv("MPM_B200_CHAIN", chain)
        case = mk(pkg, constitutive="druckerprager", gpu_precision=prec, scheme=scheme, MVL=mvl)
        dev = pkg.DeviceModel(case.args, case.grid, case.mp, case.attr, case.bc)
        dev.step(case.dt, 0.0, 24)
        out = fresh_particles(pkg, case.mp)
        dev.download(pkg._lib.F_REFERENCE | pkg._lib.F_F, out)
        dev.close()
        outs.append(out)
    agree = 1e-5 if prec == "mixed" else 1e-10
    assert rel(outs[0].xi - case.mp.xi, outs[1].xi - case.mp.xi) < agree
    for f in ("vs", "F", "Omega"):
        assert rel(getattr(outs[0], f), getattr(outs[1], f)) < agree, f
    o = orc.Oracle(case.args, case.grid, case.mp, case.attr, case.bc)
    o.run(case.dt, 0.0, 24)
    for out in outs:
        if prec == "mixed":
            check_fields(out, o, case.mp, TOL32, TOL32_STRESS)
        else:
            check_fields(out, o, case.mp, TOL64)


@pytest.mark.parametrize("prec,tol", [("fp64", TOL64), ("mixed", TOL32)])
@pytest.mark.parametrize("dim", [2, 3])
def test_mvl(pkg, orc, gpu_lib, dim, prec, tol):
    """Volumetric-locking mitigation (vollock1_OS! / vollock2_OS!,
    utils_OS.jl:1162-1257): each particle's mean stress replaced by the
    volume-weighted mean of its start-of-step cell, before the next P2G."""
    mk = small2d if dim == 2 else small3d
    case = mk(pkg, constitutive="druckerprager", gpu_precision=prec, MVL=True)
    plain = mk(pkg, constitutive="druckerprager", gpu_precision=prec)
    out, o = run_both(pkg, orc, case, 12)
    check_fields(out, o, case.mp, tol, tol_stress(tol))
    o2 = orc.Oracle(plain.args, plain.grid, plain.mp, plain.attr, plain.bc)
    o2.run(plain.dt, 0.0, 12)
    assert rel(o.sig, o2.sig) > 1e-2   # MVL changes the answer (by ~7e-2 here)


@pytest.mark.parametrize("prec,tol", [("fp64", TOL64), ("mixed", TOL32)])
@pytest.mark.parametrize("dim,va", [(2, "a"), (3, "a"), (2, "v"), (3, "v")])
def test_usl(pkg, orc, gpu_lib, dim, va, prec, tol):
    """USL (src/solvers/OS_USL.jl): no double mapping; DM1 and G2P share one
    particle pass on the device."""
    mk = small2d if dim == 2 else small3d
    case = mk(pkg, constitutive="druckerprager", gpu_precision=prec, scheme="USL", va=va,
              PIC=0.2 if va == "a" else 0.0, FLIP=0.8 if va == "a" else 1.0)
    out, o = run_both(pkg, orc, case, 12)
    check_fields(out, o, case.mp, tol, tol_stress(tol))


@pytest.mark.parametrize("prec,tol", [("fp64", TOL64), ("mixed", TOL32)])
def test_usl_mvl_graph_blocks(pkg, orc, gpu_lib, prec, tol):
    """USL with MVL over 40 steps (replayed as captured graph blocks)."""
    case = small3d(pkg, constitutive="druckerprager", gpu_precision=prec, scheme="USL", MVL=True)
    out, o = run_both(pkg, orc, case, 40)
    check_fields(out, o, case.mp, tol, tol_stress(tol))
