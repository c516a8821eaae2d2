"""Long-horizon error of the 3D slope with the lognormal cohesion field
(8 002 400 particles, 10 s): the FP32 step (FP64 positions and det F) and the
step with the stress-return surrogate, each against the all-FP64 device step,
in run-out and particle displacement at the end time.

Running the FP64 CPU oracle for 58 000 steps of 8 M particles would take
hours, so the long-horizon reference is the all-FP64 mode of the same
kernels; that mode is first validated against the oracle on a 200-step prefix
of the same slope at h = 0.2 m (1.0 M particles; the oracle's per-particle
weight tables at h = 0.1 m would need ~25 GB of host memory).

Run:  python -c "import __graft_entry__ as g; g.load_package().precision.main()" [--steps N]
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np


def _pkg():
    import __graft_entry__ as g
    return g.load_package()


def runout(x0, x):
    """Toe advance: farthest particle, and the 99.9th percentile of x (robust
    to a few ejected particles)."""
    return {"max": float(x[:, 0].max() - x0[:, 0].max()),
            "p999": float(np.percentile(x[:, 0], 99.9) - np.percentile(x0[:, 0], 99.9))}


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300))


def run_device(pkg, case, nsteps, chunk=2000, surrogate=None, log=None):
    """Step the case on the GPU; returns (positions, seconds, stats, logged samples)."""
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
    out = pkg.types.Particle3D(dx=case.mp.dx, dy=case.mp.dy, dz=case.mp.dz, xi=case.mp.xi, rho=case.mp.rho)
    dev.download(pkg._lib.F_REFERENCE, out)
    st = dev.stats()
    dev.close()
    return out, secs, st, samples


def validate_fp64_prefix(pkg, steps=200):
    from oracle import oracle as orc
    orc.build()
    case = pkg.workloads.slope_3d(h=0.2, gpu_precision="fp64", Te=0.0)
    out, secs, _, _ = run_device(pkg, case, steps)
    nth = len(os.sched_getaffinity(0))
    o = orc.Oracle(case.args, case.grid, case.mp, case.attr, case.bc, nthreads=nth)
    t0 = time.perf_counter()
    o.run(case.dt, 0.0, steps)
    t_orc = time.perf_counter() - t0
    return {"particles": int(case.mp.np), "steps": steps, "h": 0.2, "Te": 0.0,
            "disp_rel": rel(out.xi - case.mp.xi, o.xi - case.mp.xi), "stress_rel": rel(out.sig, o.sig),
            "oracle_s": t_orc, "oracle_threads": nth}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=0, help="0 = the full 10 s")
    ap.add_argument("--prefix", type=int, default=200)
    ap.add_argument("--out", default="")
    a = ap.parse_args(argv)
    pkg = _pkg()
    rep = {"workload": "3D slope, lognormal cohesion field (mean 10 kPa, CoV 0.3, 2 m), DP 25 deg"}
    rep["fp64_vs_oracle_prefix"] = validate_fp64_prefix(pkg, a.prefix)
    print(json.dumps(rep["fp64_vs_oracle_prefix"]), flush=True)
    base = pkg.workloads.slope_3d(field=True)
    nsteps = a.steps or base.nsteps_full
    rep["particles"] = int(base.mp.np)
    rep["steps"] = nsteps
    rep["t_end_s"] = nsteps * base.dt
    x0 = base.mp.xi.copy()
    res = {}
    c64 = pkg.workloads.slope_3d(gpu_precision="fp64")
    res["fp64"] = run_device(pkg, c64, nsteps)
    print("fp64 done", res["fp64"][1], flush=True)
    c32 = pkg.workloads.slope_3d(gpu_precision="mixed")
    res["mixed"] = run_device(pkg, c32, nsteps, log={"cap": 6_000_000, "every": 8})
    print("mixed done", res["mixed"][1], flush=True)
    f, y = res["mixed"][3]
    sur = pkg.surrogate.Surrogate(seed=1)
    sur.set_norm(f, y)
    t0 = time.perf_counter()
    sur.train(f, y, epochs=6, batch=16384, lr=3e-3, lr_end=1e-4)
    t_train = time.perf_counter() - t0
    cs = pkg.workloads.slope_3d(gpu_precision="mixed")
    res["surrogate"] = run_device(pkg, cs, nsteps, surrogate=sur)
    print("surrogate done", res["surrogate"][1], flush=True)
    ref_x = res["fp64"][0].xi
    ro_ref = runout(x0, ref_x)
    rep["runout_fp64_m"] = ro_ref
    for k in ("mixed", "surrogate"):
        x = res[k][0].xi
        ro = runout(x0, x)
        rep[k] = {"seconds": res[k][1], "runout_m": ro,
                  "runout_err": {q: abs(ro[q] - ro_ref[q]) / max(abs(ro_ref[q]), base.meta["h"]) for q in ro},
                  "disp_rel_vs_fp64": rel(x - x0, ref_x - x0)}
    st = res["surrogate"][2]
    rep["surrogate"].update(train_samples=int(f.shape[0]), train_s=t_train, rows=int(st.surr_rows),
                            accepted_fraction=1.0 - st.surr_fallbacks / max(st.surr_rows, 1))
    rep["surrogate"]["disp_rel_vs_mixed"] = rel(res["surrogate"][0].xi - x0, res["mixed"][0].xi - x0)
    rep["fp64"] = {"seconds": res["fp64"][1]}
    txt = json.dumps(rep)
    print(txt)
    if a.out:
        with open(a.out, "w") as fh:
            fh.write(txt + "\n")
    return rep


if __name__ == "__main__":
    main()
