"""Physical validation (not parity): the reference's 2D granular column case
(test/validation/2d_case.jl -- a 0.2 x 0.1 m sand column, Drucker-Prager
φ = 19.8°, 1 s) run through materialpointsolver on the device, its final free
surface against the laboratory surface MaterialPointSolver.jl ships for that
case (tests/golden/collapse_2d_experiment.json, made by make_collapse_experiment.py).

Measured on B200: mean |Δh| 1.0 mm over 0 <= x < 0.4 m (heights up to 100 mm),
max 2.9 mm, in both the FP64 and the mixed mode."""
import json
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "collapse_2d_experiment.json")


def experiment():
    with open(GOLDEN) as fh:
        d = json.load(fh)
    return np.array(d["surface"]), np.array(d["failure"])


def toe(x, h, level):
    """First x at which the profile h(x) falls below `level`."""
    below = np.nonzero(h < level)[0]
    if len(below) == 0:
        return x[-1]
    k = below[0]
    if k == 0:
        return x[0]
    return x[k - 1] + (x[k] - x[k - 1]) * (h[k - 1] - level) / (h[k - 1] - h[k])


def test_experiment_fixture():
    surf, fail = experiment()
    assert surf.shape == (23, 2) and fail.shape == (9, 2)
    # the deposit slopes down from the wall; its crest keeps the column height
    assert np.all(np.diff(surf[:, 0]) > 0) and np.all(np.diff(surf[:, 1]) <= 1e-3)
    assert abs(surf[0, 1] - 0.1) < 2e-3 and surf[-1, 1] < 2e-3


def test_free_surface_helper(pkg):
    xi = np.array([[0.005, 0.02], [0.006, 0.05], [0.015, 0.01], [0.035, 0.0]])
    h = pkg.workloads.free_surface(xi, np.array([0.0, 0.01, 0.02, 0.03]))
    assert h[0] == 0.05 and h[1] == 0.01 and np.isnan(h[2])


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_column_collapse_matches_experiment(pkg, gpu_lib, prec, tmp_path):
    c = pkg.workloads.collapse_2d_validation(gpu_precision=prec, project_path=str(tmp_path))
    pkg.materialpointsolver(c.args, c.grid, c.mp, c.attr, c.bc)
    surf, _ = experiment()
    edges = np.arange(0.0, 0.5 + 1e-9, 0.01)
    xc = 0.5 * (edges[1:] + edges[:-1])
    h = pkg.workloads.free_surface(c.mp.xi, edges)
    he = np.interp(xc, surf[:, 0], surf[:, 1], right=0.0)
    inner = xc < 0.4
    assert not np.isnan(h[inner]).any()
    dh = np.abs(h - he)[inner]
    assert dh.mean() < 2.5e-3, dh.mean()
    assert dh.max() < 6e-3, dh.max()
    # toe of the deposit (where the surface falls below 5 mm, four particle
    # layers; thinner tails are one or two scattered layers) within 5 cm
    h0 = np.nan_to_num(h, nan=0.0)
    assert abs(toe(xc, h0, 5e-3) - toe(surf[:, 0], surf[:, 1], 5e-3)) < 0.05
    # the column's crest stays at the wall (x < 2 cm keeps ~ the initial height)
    assert abs(h[0] - 0.1) < 3e-3


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_saturated_column_consolidates_to_hydrostatic(pkg, gpu_lib, prec, tmp_path):
    """Two-phase (coupling = :TS) physics: a 0.05 x 0.2 m saturated column,
    laterally confined, impermeable floor, settles under gravity (0.3 s with
    5 % damping of both phases).  At rest the pore pressure is hydrostatic,
    dσw/dd = -ρw g, and the skeleton carries the buoyant weight, dσ'yy/dd =
    -((1 - n) ρs + n ρw - ρw) g, with the lateral effective stress at the
    confined-elastic ratio ν / (1 - ν).  Measured on B200 in FP64: -9835 vs
    -9810 Pa/m for the water and -11322 vs -11331 Pa/m for the skeleton."""
    c = pkg.workloads.saturated_column(dim=2, h=0.01, size=(0.05, 0.2), k=0.1, Te=0.01, zeta_s=0.05,
                                       zeta_w=0.05, Ttol=0.3, gpu_precision=prec, project_path=str(tmp_path))
    pkg.materialpointsolver(c.args, c.grid, c.mp, c.attr, c.bc)
    g, n, rho_s, rho_w, nu = 9.81, c.meta["n"], 2650.0, c.meta["rho_w"], 0.3
    d = c.meta["height"] - c.mp.xi[:, 1]
    inner = d > 0.03                      # below the loosely packed top layers
    A = np.vstack([d[inner], np.ones(inner.sum())]).T

    def slope(v):
        return np.linalg.lstsq(A, v[inner], rcond=None)[0][0]

    sw, syy, sxx = slope(c.mp.sigw), slope(c.mp.sig[:, 1]), slope(c.mp.sig[:, 0])
    assert abs(sw / (-rho_w * g) - 1) < 0.02, sw
    buoyant = -((1 - n) * rho_s + n * rho_w - rho_w) * g
    assert abs(syy / buoyant - 1) < 0.02, syy
    assert abs(sxx / syy - nu / (1 - nu)) < 0.05, sxx / syy
    assert np.abs(c.mp.vs).max() < 0.02 and np.abs(c.mp.vw).max() < 0.05
