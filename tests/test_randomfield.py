"""Random fields (grf_gc! / grf_ec!, src/toolkits/randomfield.jl:57-150).

CPU: the harmonic sampling reproduces the target covariance (Gaussian:
C(r) = exp(-r^2 / lf^2), lf = 1.128379 * If), the rescalings, the lognormal
transform.  GPU: mpm_grf_eval equals an FP64 numpy evaluation of the same sum.
"""
import math

import numpy as np
import pytest


def eval_numpy(pts, H, scale):
    """scale * sum_j (a_j sin(V_j.p) + b_j cos(V_j.p)), harmonics in order."""
    pts = np.asarray(pts, float)
    if pts.shape[1] == 2:
        pts = np.column_stack([pts, np.zeros(len(pts))])
    Y = np.zeros(len(pts))
    for V1, V2, V3, a, b in H:
        t = pts[:, 0] * V1 + pts[:, 1] * V2 + pts[:, 2] * V3
        Y += a * np.sin(t) + b * np.cos(t)
    return Y * scale


def test_gc_covariance(pkg):
    """The sampled wavevectors are sqrt(2)/lf times a standard normal vector,
    so E[cos(V.r)] = exp(-r^2 / lf^2)."""
    rf = pkg.randomfield
    If = 2.0
    H = rf.harmonics_gc(np.random.default_rng(5), If=If, Nh=4000)
    lf = 1.128379 * If
    var = (H[:, :3] ** 2).mean(axis=0)
    assert np.allclose(var, 2.0 / lf ** 2, rtol=0.08)
    for r in (0.5 * If, If, 2.0 * If):
        d = np.array([r, 0.0, 0.0])
        emp = np.cos(H[:, :3] @ d).mean()
        assert emp == pytest.approx(math.exp(-r * r / lf ** 2), abs=0.04)
    assert abs(H[:, 3:].mean()) < 0.05 and abs(H[:, 3:].std() - 1.0) < 0.05


def test_ec_harmonics(pkg):
    """Exponential covariance: E[cos(V.r)] = exp(-|r|/l) along each axis."""
    H = pkg.randomfield.harmonics_ec(np.random.default_rng(6), If=(10.0, 8.0, 5.0), Nh=3000)
    for axis, L in enumerate((10.0, 8.0, 5.0)):
        d = np.zeros(3)
        d[axis] = L
        emp = np.cos(H[:, :3] @ d).mean()
        assert emp == pytest.approx(math.exp(-1.0), abs=0.05)


def test_rescale_and_lognormal(pkg):
    rf = pkg.randomfield
    Y = np.random.default_rng(2).normal(3.0, 2.0, 10000)
    m = rf._finish(Y, 5.0, 1.0, "minmax")
    assert m.min() == pytest.approx(1.0) and m.max() == pytest.approx(5.0)
    z = rf._finish(Y, 0, 1, "standard")
    assert abs(z.mean()) < 1e-12 and z.std() == pytest.approx(1.0)
    c = rf.lognormal(np.random.default_rng(3).standard_normal(400000), 10e3, 0.3)
    assert c.mean() == pytest.approx(10e3, rel=0.01)
    assert c.std() / c.mean() == pytest.approx(0.3, rel=0.02)


def test_slope_geometry(pkg):
    """The slope builder fills crest + face: 50 m^2 cross-section x 20 m at
    8 000 particles per m^3 -> about 8.0 M particles."""
    W = pkg.workloads
    pts = W.slope_points_3d(0.1, 2, 6.0, 4.05, 35.0, 20.0, np.random.default_rng(1))
    area = 6.0 * 4.05 + 0.5 * 6.0 * 6.0 / math.tan(math.radians(35.0))
    assert pts.shape[0] == pytest.approx(area * 20.0 * 8000, rel=0.01)
    tb = math.tan(math.radians(35.0))
    # the jitter (0.1 h per axis) is applied after the lattice is clipped
    assert np.all(pts[:, 0] <= 4.05 + (6.0 - pts[:, 2]) / tb + 0.03)


@pytest.mark.gpu
@pytest.mark.parametrize("dim", [2, 3])
def test_grf_eval_matches_numpy(pkg, gpu_lib, dim):
    rf = pkg.randomfield
    rng = np.random.default_rng(11)
    pts = rng.uniform(0.0, 100.0, size=(20000, dim))
    H = rf.harmonics_gc(rng, If=2.0, Nh=700)
    got = rf.evaluate(pts, H, 1.0 / math.sqrt(700))
    ref = eval_numpy(pts, H, 1.0 / math.sqrt(700))
    assert np.abs(got - ref).max() < 1e-9 * np.abs(ref).max()


@pytest.mark.gpu
def test_grf_gc_entry(pkg, gpu_lib):
    rf = pkg.randomfield
    pts = np.random.default_rng(12).uniform(0.0, 10.0, size=(5000, 3))
    Y = np.empty(5000)
    rf.grf_gc(Y, pts, 2.0, 7.0, If=1.0, Nh=500, seed=3)
    assert Y.min() == pytest.approx(2.0) and Y.max() == pytest.approx(7.0)
    H = rf.harmonics_gc(np.random.Generator(np.random.PCG64(3)), If=1.0, Nh=500)
    ref = rf._finish(eval_numpy(pts, H, 1.0 / math.sqrt(500)), 2.0, 7.0, "minmax")
    assert np.abs(Y - ref).max() < 1e-9
