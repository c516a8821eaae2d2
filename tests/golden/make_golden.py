"""Generate the golden fixtures of the tiny oracle cases.

The fixtures are produced by tests/oracle_py.py -- the pure-Python
transliteration written directly from the MaterialPointSolver.jl source, not
from oracle/ -- so that the C++ oracle is pinned to an independent reading of
the reference.  Run from the repository root:

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import __graft_entry__ as g  # noqa: E402
from oracle_py import PyModel  # noqa: E402

CASES = {
    "col2d_dp": dict(dim=2, constitutive="druckerprager", steps=4),
    "col2d_mc": dict(dim=2, constitutive="mohrcoulomb", steps=4),
    "col2d_le_pic": dict(dim=2, constitutive="linearelastic", steps=3, PIC=0.25, FLIP=0.75),
    "col3d_dp": dict(dim=3, constitutive="druckerprager", steps=3),
    "col3d_le": dict(dim=3, constitutive="linearelastic", steps=3),
    "col2d_dp_usl": dict(dim=2, constitutive="druckerprager", steps=4, scheme="USL"),
    "col3d_dp_usl_pic": dict(dim=3, constitutive="druckerprager", steps=3, scheme="USL", PIC=0.2, FLIP=0.8),
}


def tiny_case(pkg, dim, constitutive, seed=7, **extra):
    """A tiny column with random initial stress and velocity (all return-mapping
    branches get exercised within a few steps)."""
    if dim == 2:
        case = pkg.workloads.column_collapse_2d(h=0.02, width=0.06, height=0.04, domain=(0.1, 0.06),
                                                seed=seed, constitutive=constitutive, c=2000.0, **extra)
    else:
        case = pkg.workloads.column_collapse_3d(h=0.04, column=(0.08, 0.08, 0.08), domain=(0.16, 0.12, 0.12),
                                                seed=seed, constitutive=constitutive, c=2000.0, **extra)
    rng = np.random.default_rng(seed)
    case.mp.sig[:] = rng.normal(-3000.0, 2500.0, case.mp.sig.shape)
    case.mp.vs[:] = rng.normal(0.0, 0.05, case.mp.vs.shape)
    return case


def main():
    pkg = g.load_package()
    for name, spec in CASES.items():
        spec = dict(spec)
        steps = spec.pop("steps")
        case = tiny_case(pkg, spec.pop("dim"), spec.pop("constitutive"), **spec)
        m = PyModel(case.args, case.grid, case.mp, case.attr, case.bc)
        m.run(case.dt, 0.0, steps)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), xi=m.xi, vs=m.vs, sig=m.sig, eps=m.eps, F=m.F,
                            Omega=m.Omega, epsq=m.epsq, epsk=m.epsk, epsv=m.epsv, sigm=m.sigm,
                            gms=m.gms, steps=steps)
        print(name, case.mp.np, "particles", steps, "steps")


if __name__ == "__main__":
    main()
