"""Per-configuration error of the device step against the FP64 oracle (a
measurement driver for a B200, not part of the library).

For each benchmark configuration it states the relative particle-displacement
error ||Δu - Δu_ref|| / ||Δu_ref|| and the run-out error at the
configuration's horizon:

  config1  2D column, 3 200 particles, FP64, 1 s (20 657 steps): the device
           in FP64 and in the mixed mode against the CPU oracle over the whole
           run, beside the oracle's own sensitivity to its summation order
           (sequential against OpenMP atomics).
  config2  3D column, 2 560 000 particles, 1 s (22 539 steps): both device
           modes against the oracle over a 20-step prefix, then the mixed mode
           against the all-FP64 device mode over the whole second (the oracle
           would need hours), beside the run-to-run spread of each mode (the
           device reductions are atomics, so their order differs per run).
  config3  3D slope with the lognormal cohesion field (8 002 400 particles,
           10 s): the all-FP64 device mode validated against the oracle on a
           200-step prefix at h = 0.2 m, then the mixed mode and the mixed mode
           with the stress-return surrogate against it at the horizon.

Run:  python tests/precision_report.py config1|config2|config3 [--steps N] [--out FILE]
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def _pkg():
    import __graft_entry__ as g
    return g.load_package()


def _orc():
    from oracle import oracle as orc
    orc.build()
    return orc


def runout(x0, x):
    """Toe advance: farthest particle, and the 99.9th percentile of x (robust
    to a few ejected particles)."""
    return {"max": float(x[:, 0].max() - x0[:, 0].max()),
            "p999": float(np.percentile(x[:, 0], 99.9) - np.percentile(x0[:, 0], 99.9))}


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300))


def compare(x0, a, b, h):
    """Errors of run a against reference run b (dicts with xi, sig)."""
    ra, rb = runout(x0, a["xi"]), runout(x0, b["xi"])
    du = a["xi"] - b["xi"]
    return {"disp_rel": rel(a["xi"] - x0, b["xi"] - x0),
            "disp_max_over_h": float(np.abs(du).max() / h),
            "stress_rel": rel(a["sig"], b["sig"]),
            "runout_err": {q: abs(ra[q] - rb[q]) / max(abs(rb[q]), h) for q in ra}}


def run_device(pkg, case, nsteps, chunk=2000, surrogate=None, log=None):
    """Step the case on the GPU from t = 0; returns ({xi, sig}, seconds, stats, samples)."""
    dev = pkg.DeviceModel(case.args, case.grid, case.mp, case.attr, case.bc)
    if surrogate is not None:
        dev.set_surrogate(surrogate, tol=1e-3, sref=1e3)
    t0 = time.perf_counter()
    Ti, done, samples = 0.0, 0, None
    while done < nsteps:
        n = min(chunk, nsteps - done)
        if log is not None and samples is None and Ti >= case.args.Te:
            # log the first plastic steps of the plain run (the physics is unchanged)
            f, y, Ti = pkg.surrogate.collect_samples(dev, case.dt, Ti, n, log["cap"], every=log["every"])
            samples = (f, y)
        else:
            Ti = dev.step(case.dt, Ti, n)
        done += n
    secs = time.perf_counter() - t0
    if case.grid.dim == 3:
        out = pkg.types.Particle3D(dx=case.mp.dx, dy=case.mp.dy, dz=case.mp.dz, xi=case.mp.xi, rho=case.mp.rho)
    else:
        out = pkg.types.Particle2D(dx=case.mp.dx, dy=case.mp.dy, xi=case.mp.xi, rho=case.mp.rho)
    dev.download(pkg._lib.F_REFERENCE, out)
    st = dev.stats()
    dev.close()
    return {"xi": out.xi.copy(), "sig": out.sig.copy()}, secs, st, samples


def run_oracle(orc, case, nsteps, nthreads):
    o = orc.Oracle(case.args, case.grid, case.mp, case.attr, case.bc, nthreads=nthreads)
    t0 = time.perf_counter()
    o.run(case.dt, 0.0, nsteps)
    return {"xi": np.array(o.xi), "sig": np.array(o.sig)}, time.perf_counter() - t0


def config1(pkg, orc, steps=0):
    base = pkg.workloads.column_collapse_2d()
    n = steps or base.nsteps_full
    h = base.meta["h"]
    x0 = base.mp.xi.copy()
    nth = len(os.sched_getaffinity(0))
    rep = {"config": "2D column collapse, 3 200 particles, DP 19.8 deg, FP64", "steps": n, "t_end_s": n * base.dt}
    seq, t_seq = run_oracle(orc, base, n, 1)
    par, t_par = run_oracle(orc, base, n, nth)
    rep["oracle_seconds"] = {"sequential": t_seq, f"openmp_{nth}": t_par}
    rep["runout_oracle_m"] = runout(x0, seq["xi"])
    rep["oracle_openmp_vs_sequential"] = compare(x0, par, seq, h)
    for prec in ("fp64", "mixed"):
        c = pkg.workloads.column_collapse_2d(gpu_precision=prec)
        d, secs, _, _ = run_device(pkg, c, n, chunk=n)
        rep[f"device_{prec}"] = dict(compare(x0, d, seq, h), seconds=secs)
    return rep


def config2(pkg, orc, steps=0, prefix=20):
    base = pkg.workloads.column_collapse_3d()
    n = steps or base.nsteps_full
    h = base.meta["h"]
    x0 = base.mp.xi.copy()
    nth = len(os.sched_getaffinity(0))
    rep = {"config": "3D column collapse, 2 560 000 particles, Mohr-Coulomb (3D literal), mixed precision",
           "particles": int(base.mp.np), "steps": n, "t_end_s": n * base.dt}
    o, t_o = run_oracle(orc, base, prefix, nth)
    rep["prefix"] = {"steps": prefix, "oracle_seconds": t_o, "oracle_threads": nth}
    for prec in ("fp64", "mixed"):
        c = pkg.workloads.column_collapse_3d(gpu_precision=prec)
        d, _, _, _ = run_device(pkg, c, prefix)
        rep["prefix"][f"device_{prec}_vs_oracle"] = compare(x0, d, o, h)
    del o
    runs = {}
    for key, prec in (("fp64_a", "fp64"), ("fp64_b", "fp64"), ("mixed_a", "mixed"), ("mixed_b", "mixed")):
        c = pkg.workloads.column_collapse_3d(gpu_precision=prec)
        runs[key], secs, _, _ = run_device(pkg, c, n, chunk=n)
        rep.setdefault("seconds", {})[key] = secs
        print(key, secs, flush=True)
    ref = runs["fp64_a"]
    rep["runout_fp64_m"] = runout(x0, ref["xi"])
    rep["fp64_run_to_run"] = compare(x0, runs["fp64_b"], ref, h)
    rep["mixed_vs_fp64"] = compare(x0, runs["mixed_a"], ref, h)
    rep["mixed_b_vs_fp64"] = compare(x0, runs["mixed_b"], ref, h)
    rep["mixed_run_to_run"] = compare(x0, runs["mixed_b"], runs["mixed_a"], h)
    return rep


def config3(pkg, orc, steps=0, prefix=200):
    rep = {"config": "3D slope, lognormal cohesion field (mean 10 kPa, CoV 0.3, 2 m), DP 25 deg"}
    pc = pkg.workloads.slope_3d(h=0.2, gpu_precision="fp64", Te=0.0)
    d, _, _, _ = run_device(pkg, pc, prefix)
    o, t_o = run_oracle(orc, pc, prefix, len(os.sched_getaffinity(0)))
    rep["fp64_vs_oracle_prefix"] = dict(compare(pc.mp.xi, d, o, 0.2), particles=int(pc.mp.np), steps=prefix,
                                        h=0.2, oracle_seconds=t_o)
    del d, o
    print(json.dumps(rep["fp64_vs_oracle_prefix"]), flush=True)
    base = pkg.workloads.slope_3d(field=True)
    n = steps or base.nsteps_full
    h = base.meta["h"]
    rep.update(particles=int(base.mp.np), steps=n, t_end_s=n * base.dt)
    x0 = base.mp.xi.copy()
    res = {}
    res["fp64"] = run_device(pkg, pkg.workloads.slope_3d(gpu_precision="fp64"), n)
    print("fp64 done", res["fp64"][1], flush=True)
    res["mixed"] = run_device(pkg, pkg.workloads.slope_3d(gpu_precision="mixed"), n,
                              log={"cap": 6_000_000, "every": 8})
    print("mixed done", res["mixed"][1], flush=True)
    f, y = res["mixed"][3]
    sur = pkg.surrogate.Surrogate(seed=1)
    sur.set_norm(f, y)
    t0 = time.perf_counter()
    sur.train(f, y, epochs=6, batch=16384, lr=3e-3, lr_end=1e-4)
    t_train = time.perf_counter() - t0
    res["surrogate"] = run_device(pkg, pkg.workloads.slope_3d(gpu_precision="mixed"), n, surrogate=sur)
    print("surrogate done", res["surrogate"][1], flush=True)
    ref = res["fp64"][0]
    rep["runout_fp64_m"] = runout(x0, ref["xi"])
    rep["fp64"] = {"seconds": res["fp64"][1]}
    for k in ("mixed", "surrogate"):
        rep[k] = dict(compare(x0, res[k][0], ref, h), seconds=res[k][1])
    st = res["surrogate"][2]
    rep["surrogate"].update(train_samples=int(f.shape[0]), train_s=t_train, rows=int(st.surr_rows),
                            accepted_fraction=1.0 - st.surr_fallbacks / max(st.surr_rows, 1),
                            vs_mixed=compare(x0, res["surrogate"][0], res["mixed"][0], h))
    return rep


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("config", choices=["config1", "config2", "config3"])
    ap.add_argument("--steps", type=int, default=0, help="0 = the configuration's full horizon")
    ap.add_argument("--out", default="")
    a = ap.parse_args(argv)
    pkg, orc = _pkg(), _orc()
    rep = {"config1": config1, "config2": config2, "config3": config3}[a.config](pkg, orc, a.steps)
    txt = json.dumps(rep)
    print(txt)
    if a.out:
        with open(a.out, "w") as fh:
            fh.write(txt + "\n")
    return rep


if __name__ == "__main__":
    main()
