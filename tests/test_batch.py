"""Batches of independent 2D slopes packed into one grid (one launch per pass
covers every slope), and the run-time autotuner.

CPU: the drawn slopes hold the drawn particle counts, the regions of the
slopes share no grid node, the boundary layout.  GPU: every slope of a batch
moves as it does when run alone (the plain step), the batch matches the oracle,
and the autotuner's trial steps are ordinary steps of the model.
"""
import math

import numpy as np
import pytest

from helpers import fresh_particles, rel

SMALL = dict(np_range=(300.0, 1500.0), height=(1.5, 3.0), h=0.5)


def small_batch(pkg, n=4, **kw):
    W = pkg.workloads
    specs = W.draw_slope_specs(n, seed=41, **SMALL)
    base = dict(specs=specs, h=0.5, Te=0.0, Ttol=5.0)
    base.update(kw)
    return W.slope_batch_2d(**base)


def test_specs_hold_the_drawn_counts(pkg):
    W = pkg.workloads
    specs = W.draw_slope_specs(64, seed=7)
    assert all(1.0e4 <= s["target_np"] <= 2.0e5 for s in specs)
    assert all(math.radians(25) <= s["beta"] <= math.radians(45) for s in specs)
    assert all(s["H"] <= 20.0 and s["crest"] >= 0.0 for s in specs)
    for s in specs[:6]:
        pts = W.slope_points_2d(s, 0.05)
        assert len(pts) == pytest.approx(s["target_np"], rel=0.01)


def test_regions_share_no_node(pkg):
    case = small_batch(pkg, 5)
    h = case.meta["h"]
    sl = case.meta["slopes"]
    xi = case.mp.xi
    for a, b in zip(sl, sl[1:]):
        # the uGIMP stencil reaches at most 2 nodes past a particle's cell
        assert b["x0"] - (a["x0"] + a["L"]) >= 5 * h
    for k, s in enumerate(sl):
        x = xi[s["start"]:s["end"], 0]
        assert x.min() > s["x0"] and x.max() < s["x0"] + s["L"]
        assert np.all(case.attr.nid[s["start"]:s["end"]] == k + 1)
    g = case.grid
    fx = np.asarray(case.bc.vx_s_idx).reshape(g.nnx, g.nny)
    fy = np.asarray(case.bc.vy_s_idx).reshape(g.nnx, g.nny)
    assert fy[:, g._vy <= 1e-9].all() and fx[:, g._vy <= 1e-9].all()       # fixed floor
    ix0 = int(round((sl[1]["x0"] - g.x1) / h))
    assert fx[ix0].all() and not fy[ix0, g._vy > 1e-9].any()               # wall: vx only


def test_single_slope_has_the_same_particles(pkg):
    W = pkg.workloads
    case = small_batch(pkg, 3)
    for k, s in enumerate(case.meta["slopes"]):
        one = W.slope_2d_single(case, k)
        assert one.mp.np == s["np"]
        assert np.allclose(one.mp.xi[:, 0] + s["x0"], case.mp.xi[s["start"]:s["end"], 0], atol=1e-12)
        assert np.array_equal(one.mp.xi[:, 1], case.mp.xi[s["start"]:s["end"], 1])


def run_dev(pkg, case, nsteps):
    dev = pkg.DeviceModel(case.args, case.grid, case.mp, case.attr, case.bc)
    dev.step(case.dt, 0.0, nsteps)
    out = fresh_particles(pkg, case.mp)
    dev.download(pkg._lib.F_REFERENCE | pkg._lib.F_F, out)
    dev.close()
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("prec,tol", [("fp64", 1e-9), ("mixed", 1e-4)])
def test_batch_equals_plain_runs(pkg, gpu_lib, prec, tol):
    """Each slope of the batch against the same slope run alone through the
    plain step: displacement, velocity, stress; run-outs within 1e-3."""
    W = pkg.workloads
    nsteps = 40
    case = small_batch(pkg, 4, gpu_precision=prec)
    out = run_dev(pkg, case, nsteps)
    ro_batch = W.slope_runouts(case, out.xi)
    for k, s in enumerate(case.meta["slopes"]):
        one = W.slope_2d_single(case, k, gpu_precision=prec)
        o1 = run_dev(pkg, one, nsteps)
        sl = slice(s["start"], s["end"])
        du_b = out.xi[sl] - case.mp.xi[sl]
        du_1 = o1.xi - one.mp.xi
        assert rel(du_b, du_1) < tol, (k, rel(du_b, du_1))
        assert rel(out.vs[sl], o1.vs) < tol
        assert rel(out.sig[sl], o1.sig) < 10 * tol
        ro1 = W.slope_runouts(one, o1.xi)[0]
        assert abs(ro_batch[k] - ro1) <= 1e-3 * max(abs(ro1), case.meta["h"])


@pytest.mark.gpu
def test_batch_matches_oracle(pkg, orc, gpu_lib):
    case = small_batch(pkg, 3, gpu_precision="fp64")
    out = run_dev(pkg, case, 20)
    o = orc.Oracle(case.args, case.grid, case.mp, case.attr, case.bc)
    o.run(case.dt, 0.0, 20)
    assert rel(out.xi - case.mp.xi, o.xi - case.mp.xi) < 1e-9
    assert rel(out.sig, o.sig) < 1e-9
    assert np.abs(o.epsq).max() > 0


@pytest.mark.gpu
@pytest.mark.parametrize("prec,tol", [("fp64", 1e-9), ("mixed", 1e-4)])
def test_autotune_steps_are_model_steps(pkg, orc, gpu_lib, prec, tol):
    """The autotuner's trials (2 tile shapes x re-sort periods 8, 16, 32, 64 at
    max(12, period) steps each, then the fused pass at 3 CTAs per SM at periods
    32 and 64, then the tiled and the box passes at periods 16 and 32, then the
    two finalists again, 64 steps each) are 568 ordinary steps: the state
    equals the oracle's after 568 steps (in the mixed mode through every
    variant and tile shape), and the chosen tuning is one of the candidates and
    stays set."""
    case = small_batch(pkg, 3, gpu_precision=prec)
    dev = pkg.DeviceModel(case.args, case.grid, case.mp, case.attr, case.bc)
    Ti, S, tiled, ms = dev.autotune(case.dt, 0.0, 12)
    nsteps = 2 * (12 + 16 + 32 + 64) + (32 + 64) + 2 * (16 + 32) + 2 * 64
    assert nsteps == 568
    assert S in (8, 16, 32, 64) and tiled in (0, 1, 2, 3) and len(ms) == 16 and all(m > 0 for m in ms)
    assert dev.tuning() == (S, tiled)
    assert dev.tile() in ((4, 8, 1), (2, 16, 1))
    assert Ti == pytest.approx(nsteps * case.dt, rel=1e-12)
    assert dev.stats().steps_done == nsteps
    out = fresh_particles(pkg, case.mp)
    dev.download(pkg._lib.F_REFERENCE, out)
    dev.close()
    o = orc.Oracle(case.args, case.grid, case.mp, case.attr, case.bc)
    o.run(case.dt, 0.0, nsteps)
    assert rel(out.xi - case.mp.xi, o.xi - case.mp.xi) < tol
    assert rel(out.sig, o.sig) < (tol if prec == "fp64" else 1e-3)
