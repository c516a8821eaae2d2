"""The FP64 oracle (oracle/) against hand-derived known answers, against the
independent pure-Python transliteration of the reference (tests/oracle_py.py)
and against the golden fixtures that transliteration produced
(tests/golden/make_golden.py).  CPU only."""
import math
import os

import numpy as np
import pytest

from golden.make_golden import CASES, tiny_case
from oracle_py import PyModel, fld as py_fld, cld as py_cld
from helpers import rel

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


# ---- uGIMP basis, mpbasisfunc.jl:40-53: hand-derived values (h = 1, lp = 0.5) ----
@pytest.mark.parametrize("d,N,dN", [
    (0.0, 0.875, 0.0),            # 1 - (0 + lp^2)/(4 h lp)
    (0.1, 1 - (0.04 + 0.25) / 2.0, -0.4),
    (0.25, 0.75, -1.0),           # region 2 starts at lp/2
    (-0.5, 0.5, 1.0),
    (0.75, 0.25, -1.0),           # region 3 starts at h - lp/2: (1.25 - 0.75)^2 / (2 h lp)
    (1.0, 0.0625, -0.5),
    (1.25, 0.0, 0.0),             # support ends at h + lp/2 (open)
    (-1.3, 0.0, 0.0),
])
def test_ugimp_known_values(orc, d, N, dN):
    n, dn = orc.ugimp(d, 1.0, 0.5)
    assert n == pytest.approx(N, abs=1e-15)
    assert dn == pytest.approx(dN, abs=1e-15)


@pytest.mark.parametrize("lp", [0.25, 0.5, 1.0])
def test_ugimp_partition_of_unity(orc, lp):
    for s in np.linspace(0.0, 0.999, 37):
        w = [orc.ugimp(s - j, 1.0, lp) for j in (-1, 0, 1, 2)]
        assert sum(x[0] for x in w) == pytest.approx(1.0, abs=1e-14)
        assert sum(x[1] for x in w) == pytest.approx(0.0, abs=1e-14)


# ---- Julia float fld / cld: the exact-remainder rule ----
def test_fld_cld_known_values(orc):
    assert orc.fld(1.0, 0.1) == 9.0          # 0.1 is slightly above 1/10: floor(1.0/0.1) would give 10
    assert math.floor(1.0 / 0.1) == 10
    assert orc.cld(1.0, 0.1) == 10.0
    assert orc.fld(-1e-20, 0.005) == -1.0
    assert orc.cld(1e-20, 0.005) == 1.0
    assert orc.fld(0.0, 0.005) == 0.0 and orc.cld(0.0, 0.005) == 0.0
    assert orc.fld(0.015, 0.005) == 2.0 and orc.cld(0.015, 0.005) == 3.0
    rng = np.random.default_rng(1)
    for a, b in zip(rng.normal(0, 3, 400), rng.uniform(0.001, 0.5, 400)):
        assert orc.fld(a, b) == py_fld(a, b)
        assert orc.cld(a, b) == py_cld(a, b)


def test_p2c_on_node_lines(pkg, orc):
    """Particles exactly on node lines: y belongs to the lower cell (cld), x and z
    to the upper one (fld); ids are 1-based (utils_OS.jl:247-249, 380-383)."""
    case = pkg.workloads.column_collapse_3d(h=0.04, column=(0.08, 0.08, 0.08), domain=(0.16, 0.12, 0.12))
    g = case.grid
    o = orc.Oracle(case.args, g, case.mp, case.attr, case.bc)
    # node (ix=3, iy=4, iz=5) exactly
    x = np.array([[g.x1 + 3 * g.dx, g.y1 + 4 * g.dy, g.z1 + 5 * g.dz]])
    p = o.p2c(x)[0]
    cx = int(py_fld(x[0, 0] - g.x1, g.dx))
    cy = int(py_cld(x[0, 1] - g.y1, g.dy))
    cz = int(py_fld(x[0, 2] - g.z1, g.dz))
    assert p == cy + cz * g.ncy * g.ncx + cx * g.ncy


# ---- single-particle Drucker-Prager return, druckerprager.jl:89-155 ----
def dp_expected(s, K, G, c, phi, psi, st):
    sm = (s[0] + s[1] + s[2]) * 0.333333
    sij = np.array(s, float); sij[:3] -= sm
    tau = math.sqrt(0.5 * (sij[0] ** 2 + sij[1] ** 2 + sij[2] ** 2) + sij[3] ** 2 + sij[4] ** 2 + sij[5] ** 2)
    kphi = 6 * c * math.cos(phi) / (1.732051 * (3 + math.sin(phi)))
    qphi = 6 * math.sin(phi) / (1.732051 * (3 + math.sin(phi)))
    qpsi = 6 * math.sin(psi) / (1.732051 * (3 + math.sin(psi)))
    st = min(st, kphi / qphi)
    return sm, sij, tau, kphi, qphi, qpsi, st


def test_dp_elastic_shear_tension(orc):
    K, G, c, phi, psi = 7e5, 3.2e5, 1000.0, math.radians(30), math.radians(5)
    # elastic: mild compression, small deviator
    s, q, k = orc.dp_point(3, [-1e4, -1e4, -1e4, 100, 0, 0], 0, 0, K, G, c, phi, psi, 0.0)
    assert np.allclose(s, [-1e4, -1e4, -1e4, 100, 0, 0]) and q == 0 and k == 0
    # shear: large deviator under compression -> back onto the cone, fs = 0 afterwards
    s0 = [-2e4, -1e4, -1.5e4, 8e3, 2e3, -1e3]
    s, q, k = orc.dp_point(3, s0, 0, 0, K, G, c, phi, psi, 0.0)
    sm, sij, tau, kphi, qphi, qpsi, st = dp_expected(s0, K, G, c, phi, psi, 0.0)
    fs = tau + qphi * sm - kphi
    dl = fs / (G + K * qphi * qpsi)
    t1 = sm - K * qpsi * dl
    t2 = (kphi - qphi * t1) / tau
    exp = np.r_[sij[:3] * t2 + t1, sij[3:] * t2]
    assert np.allclose(s, exp, rtol=1e-12)
    assert q == pytest.approx(dl * math.sqrt(0.333333 + 0.222222 * qpsi ** 2), rel=1e-12)
    sm2, sij2, tau2, *_ = dp_expected(s, K, G, c, phi, psi, 0.0)
    assert tau2 + qphi * sm2 - kphi == pytest.approx(0.0, abs=1e-6 * kphi + 1e-3)
    # tension: mean stress above the cut-off with a small deviator
    s0 = [3e3, 3e3, 3e3, 10, 0, 0]
    s, q, k = orc.dp_point(3, s0, 0, 0, K, G, c, phi, psi, 500.0)
    sm, sij, tau, kphi, qphi, qpsi, st = dp_expected(s0, K, G, c, phi, psi, 500.0)
    assert np.allclose(s[:3], sij[:3] + st) and np.allclose(s[3:], s0[3:])
    assert k == pytest.approx((sm - st) / K, rel=1e-12)


def _mc_yield(s, c, phi, st):
    s = np.asarray(s, float)
    sm = s[:3].mean()
    dev = s.copy(); dev[:3] -= sm
    j2 = ((s[0] - s[1]) ** 2 + (s[1] - s[2]) ** 2 + (s[2] - s[0]) ** 2) / 6 + s[3] ** 2 + s[4] ** 2 + s[5] ** 2
    j3 = dev[0] * dev[1] * dev[2] + 2 * s[3] * s[4] * s[5] - dev[0] * s[4] ** 2 - dev[1] * s[5] ** 2 - dev[2] * s[3] ** 2
    th = math.acos(max(-1.0, min(1.0, 1.5 * math.sqrt(3) * j3 / j2 ** 1.5))) / 3
    rho, eps = math.sqrt(2 * j2), math.sqrt(3) * sm
    ft = math.sqrt(2 / 3) * math.cos(th) * rho + eps / math.sqrt(3) - st
    fs = (math.sqrt(1.5) * rho * (math.sin(th + math.pi / 3) / (math.sqrt(3) * math.cos(phi)) +
                                  math.cos(th + math.pi / 3) * math.tan(phi) / 3) + eps / math.sqrt(3) * math.tan(phi) - c)
    return ft, fs


@pytest.mark.parametrize("scale", [10.0, 40.0])
def test_mc3d_restated_returns_to_surface(orc, scale):
    """The restated 3D Mohr-Coulomb brings a yielding trial state back inside the
    surface (both yield functions below the 0.1 tolerance afterwards) and
    accumulates plastic strain."""
    K, G, c, phi, psi, st = 8.3e5, 3.8e5, 500.0, math.radians(30), 0.0, 0.0
    sig0 = np.array([-1e4, -1e4, -1e4, 0, 0, 0])
    de = scale * np.array([-2e-3, 1e-3, 0.0, 4e-3, 0.0, 0.0])
    Dt, Dd = K + 4 * G / 3, K - 2 * G / 3
    trial = sig0 + np.array([Dt * de[0] + Dd * (de[1] + de[2]), Dt * de[1] + Dd * (de[0] + de[2]),
                             Dt * de[2] + Dd * (de[0] + de[1]), G * de[3], G * de[4], G * de[5]])
    ft, fs = _mc_yield(trial, c, phi, st)
    assert max(ft, fs) > 0
    s, q = orc.mc3d_point(trial, sig0, de, 0.0, K, G, c, phi, psi, st)
    assert q > 0
    ft, fs = _mc_yield(s, c, phi, st)
    assert ft < 0.1 and fs < 0.1


# ---- the C++ oracle against the independent transliteration ----
@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_transliteration(pkg, orc, name):
    spec = dict(CASES[name])
    steps = spec.pop("steps")
    case = tiny_case(pkg, spec.pop("dim"), spec.pop("constitutive"), **spec)
    o = orc.Oracle(case.args, case.grid, case.mp, case.attr, case.bc)
    o.run(case.dt, 0.0, steps)
    m = PyModel(case.args, case.grid, case.mp, case.attr, case.bc)
    m.run(case.dt, 0.0, steps)
    for f in ("xi", "vs", "sig", "eps", "F", "Omega", "epsq", "epsk", "epsv", "sigm"):
        assert rel(getattr(o, f), getattr(m, f)) < 1e-12, f
    assert rel(o.g_ms, m.gms) < 1e-12


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_golden(pkg, orc, name):
    spec = dict(CASES[name])
    steps = spec.pop("steps")
    case = tiny_case(pkg, spec.pop("dim"), spec.pop("constitutive"), **spec)
    gold = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    assert int(gold["steps"]) == steps
    o = orc.Oracle(case.args, case.grid, case.mp, case.attr, case.bc)
    o.run(case.dt, 0.0, steps)
    for f in ("xi", "vs", "sig", "eps", "F", "Omega", "epsq", "epsk", "epsv", "sigm"):
        assert rel(getattr(o, f), gold[f]) < 1e-12, f


def test_oracle_threads_match_sequential(pkg, orc):
    """OpenMP mode (the timed CPU baseline) computes the sequential result up to
    the summation order of its atomics."""
    case = tiny_case(pkg, 3, "druckerprager")
    a = orc.Oracle(case.args, case.grid, case.mp, case.attr, case.bc, nthreads=0)
    b = orc.Oracle(case.args, case.grid, case.mp, case.attr, case.bc, nthreads=4)
    a.run(case.dt, 0.0, 3)
    b.run(case.dt, 0.0, 3)
    assert rel(a.xi - case.mp.xi, b.xi - case.mp.xi) < 1e-10
    assert rel(a.sig, b.sig) < 1e-10


def test_mc3d_literal_is_elastic(pkg, orc):
    """The reference's 3D mcP! body is commented out: 3D "mohrcoulomb" equals
    linear elasticity in literal mode."""
    ca = tiny_case(pkg, 3, "mohrcoulomb")
    cb = tiny_case(pkg, 3, "linearelastic")
    a = orc.Oracle(ca.args, ca.grid, ca.mp, ca.attr, ca.bc)
    b = orc.Oracle(cb.args, cb.grid, cb.mp, cb.attr, cb.bc)
    a.run(ca.dt, 0.0, 3)
    b.run(cb.dt, 0.0, 3)
    assert np.array_equal(a.sig, b.sig) and np.array_equal(a.xi, b.xi)
