#!/usr/bin/env python
"""Benchmark: explicit uGIMP MPM steps on the 3D granular column collapse.

Workload (per GPU): 3D column collapse, domain 1.2 x 0.4 x 0.6 m, h = 5 mm,
column 0.5 x 0.2 x 0.4 m at 2x2x2 particles per cell = 2 560 000 particles,
Mohr-Coulomb (phi = 30 deg, c = 0, psi = 0), rho = 2650, E = 1 MPa, nu = 0.3,
free-slip walls, CFL 0.2, FP32 bulk with FP64 positions and det(F).  A bench
step is one MPM time step over all particles (cell re-sort every 32 steps
included).  The particle state (~0.5 GB) exceeds the 126 MB L2, so no flush is
needed between steps.

Metric: particle-updates/s = particles x steps / device time (max over ranks).
Multi-GPU runs are independent replicas (the reference has no multi-GPU path):
value = sum of particles x steps over ranks / max time, scaling "weak".

--impl reference times the CPU restatement of the reference's path
(oracle/, OpenMP on all host cores) on the same workload, one MPM step per
bench step.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extra", action="store_true",
                    help="column3d: skip the batched (batch2d) and learned (slope3d surrogate) forms")
    ap.add_argument("--mc3d", default="literal", choices=["literal", "restated"])
    ap.add_argument("--workload", default="column3d",
                    choices=["column3d", "slope3d", "batch2d", "column2d", "saturated3d", "example3d", "example2d"],
                    help="column3d: the 2.56 M-particle 3D column (the headline); slope3d: the 8.0 M-particle "
                         "3D slope with a lognormal cohesion field; batch2d: 256 independent 2D slopes "
                         "(15.5 M particles) advanced together, autotuned during warm-up; column2d: the 3 200-"
                         "particle 2D column in FP64 (launch-bound; CUDA graph replay); saturated3d: the 2.56 M-particle column "
                         "as a two-phase (solid + water) saturated soil, coupling TS; example3d: the reference's "
                         "own 3D example (512 000 particles, MVL on), against its published 66.3 it/s; example2d: its "
                         "2D example (20 000 particles), against its published 2.11e3 it/s")
    ap.add_argument("--surrogate", action="store_true",
                    help="slope3d: train the stress-return surrogate on samples logged from plain steps "
                         "(untimed) and time steps with it")
    ap.add_argument("--snapshot-every", type=int, default=0,
                    help="also time K steps with an HDF5 snapshot group every N steps (submit_work!'s "
                         "hdf5 branch) against the same chunks without snapshots")
    ap.add_argument("--profile-run", action="store_true",
                    help="only W warm-up + K device steps (the command profilers wrap)")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled through NVML
    (read-only queries) every 5 ms while the timed region runs, plus one
    sample right before and one right after it, so that even a region of a
    few milliseconds has a record.  Falls back to nvidia-smi polling when
    NVML is not available."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index):
        self.index = index
        self.rows = []          # (sm_mhz, max_mhz, set of reasons)
        self.proc = None
        self.nv = None
        self.stop = threading.Event()

    def _nvml_handle(self):
        import pynvml as nv
        nv.nvmlInit()
        self.nv = nv
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(self.index).uuid)
            return nv.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            return nv.nvmlDeviceGetHandleByIndex(self.index)

    def _sample(self):
        nv = self.nv
        sm = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
        mx = nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM)
        bits = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
        masks = [nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                 nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap]
        self.rows.append((float(sm), float(mx), {n for n, m in zip(self.NAMES, masks) if bits & m}))

    def _poll(self):
        while not self.stop.wait(0.005):
            try:
                self._sample()
            except Exception:
                return

    def __enter__(self):
        try:
            self.h = self._nvml_handle()
            self._sample()
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
        except Exception:
            self.nv = None
            try:
                self.proc = subprocess.Popen(
                    ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                     "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
                self.t = threading.Thread(target=self._read, daemon=True)
                self.t.start()
            except OSError:
                self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            r = [x.strip() for x in line.split(",")]
            try:
                reasons = {n for k, n in enumerate(self.NAMES) if len(r) > 5 + k and r[5 + k].lower() == "active"}
                self.rows.append((float(r[1]), float(r[2]), reasons))
            except ValueError:
                pass

    def __exit__(self, *a):
        if self.nv is not None:
            self.stop.set()
            self.t.join(timeout=2)
            try:
                self._sample()
            except Exception:
                pass
        elif self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.t.join(timeout=2)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        reasons = set()
        for r in self.rows:
            reasons |= r[2]
        return {"sm_mhz": statistics.median(r[0] for r in self.rows),
                "sm_max_mhz": max(r[1] for r in self.rows),
                "reasons": sorted(reasons), "samples": len(self.rows),
                "source": "nvml" if self.nv is not None else "nvidia-smi"}


def max_over_ranks(x, device):
    """Max of a per-rank scalar over all ranks of the default process group."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(world, npart, steps, t_max_ms):
    """Whole-job particle-updates/s of `world` independent replicas, each
    stepping `npart` particles `steps` times, timed by the slowest rank."""
    return world * npart * steps / (t_max_ms * 1e-3)


WORKLOADS = {
    "column3d": {"workload": "3D granular column collapse, uGIMP, MUSL va=:a", "constitutive": "mohrcoulomb"},
    "slope3d": {"workload": "3D slope failure with a lognormal cohesion field, uGIMP, MUSL va=:a",
                "constitutive": "druckerprager"},
    "batch2d": {"workload": "256 independent 2D slopes in one grid, uGIMP, MUSL va=:a",
                "constitutive": "druckerprager"},
    "column2d": {"workload": "2D granular column collapse (3 200 particles), uGIMP, MUSL va=:a, all FP64",
                 "constitutive": "druckerprager"},
    "saturated3d": {"workload": "3D saturated soil column collapse, two-phase (coupling TS), uGIMP, MUSL",
                    "constitutive": "druckerprager"},
    "example3d": {"workload": "the reference's 3D column-collapse example (examples/3d_collapse.ipynb), uGIMP, "
                              "MUSL va=:a, MVL on", "constitutive": "druckerprager"},
    "example2d": {"workload": "the reference's 2D column-collapse example (examples/2d_collapse.ipynb), uGIMP, "
                              "MUSL va=:a", "constitutive": "druckerprager"},
}

# The reference's published throughput for the example3d case: 66.3 it/s with
# 512 000 particles, FP64, on an unstated NVIDIA GPU (examples/3d_collapse.ipynb:381).
EXAMPLE3D_PUBLISHED = 66.3 * 512000
# ... and for the example2d case: 2.11e3 it/s with 20 000 particles, FP64, on an
# unstated NVIDIA GPU (examples/2d_collapse.ipynb:385).
EXAMPLE2D_PUBLISHED = 2.11e3 * 20000
EXAMPLES = {"example3d": ("collapse_3d_example", EXAMPLE3D_PUBLISHED,
                          "examples/3d_collapse.ipynb:381: 66.3 it/s x 512 000 particles, FP64, unstated NVIDIA GPU"),
            "example2d": ("collapse_2d_example", EXAMPLE2D_PUBLISHED,
                          "examples/2d_collapse.ipynb:385: 2.11e3 it/s x 20 000 particles, FP64, unstated NVIDIA GPU")}


PASS_VARIANTS = {0: "lane-merged per-particle", 1: "tiled", 2: "box",
                 3: "lane-merged per-particle, fused pass at 3 CTAs/SM"}


def make_case(mc3d, workload="column3d", surrogate=False):
    import __graft_entry__ as g
    pkg = g.load_package()
    if workload == "slope3d":
        # the run starts in the plastic regime (no gravity ramp: during the
        # ramp Ti < Te the reference skips the return mapping), so that the
        # timed steps carry the Drucker-Prager return -- and, with the
        # surrogate, the return it replaces
        case = pkg.workloads.slope_3d(Te=0.0)
    elif workload == "batch2d":
        case = pkg.workloads.slope_batch_2d(Te=0.0)   # plastic regime, as above
    elif workload == "column2d":
        case = pkg.workloads.column_collapse_2d(gpu_precision="fp64")
    elif workload in EXAMPLES:
        case = getattr(pkg.workloads, EXAMPLES[workload][0])()
    elif workload == "saturated3d":
        case = pkg.workloads.saturated_column(dim=3, h=0.005, size=(0.5, 0.2, 0.4), box=(1.2, 0.4, 0.6),
                                              constitutive="druckerprager", seed=1002)
    else:
        case = pkg.workloads.column_collapse_3d(mc3d=mc3d)
    return pkg, case


def pin_particles(mp):
    """Move the particle arrays into page-locked host memory (torch pinned
    buffers viewed as numpy) so host<->device copies run at full PCIe rate."""
    try:
        import torch
    except ImportError:
        return
    names = ["xi", "vs", "sig", "eps", "epsq", "epsk", "epsv", "Omega", "Omega0", "rho", "rho0", "F", "ms", "sigm"]
    if getattr(mp, "phase", 1) == 2:
        names += ["n", "rho_w", "sigw", "vw", "epsw", "mw"]
    for name in names:
        a = getattr(mp, name)
        t = torch.empty(a.size, dtype=getattr(torch, str(a.dtype)), pin_memory=True)
        b = t.numpy()
        if a.ndim == 2:
            b = b.reshape(a.shape[1], a.shape[0]).T   # column-major view
        b[...] = a
        setattr(mp, name + "_pinned_owner", t)
        setattr(mp, name, b)


G2P_TRAFFIC_PER_PARTICLE = 250.9   # B, dram__bytes_read.sum + dram__bytes_write.sum / np

# algorithmic bytes per particle / per active node
BP_STEP_3D = 212       # particle state read + written once per step
BN_STEP_3D = 156       # compulsory grid traffic per active node per step
BP_G2P_3D = 200        # fused G2P+stress+P2G kernel: its own particle bytes
BN_G2P_3D = 40         # Δu read (3 floats) + m, p, f written (7 floats)
# two-phase: the water phase's particle fields (n, σw, mw, vw, ϵijw read; n, σw,
# vw, ϵijw written) and node records (Δus, Δuw, vsT read; ms, ps, fs, mi, mw,
# pw, fw, fd written in the fused pass; all the water records in the step)
BP_STEP_TS = 304
BN_STEP_TS = 344
BP_G2P_TS = 280
BN_G2P_TS = 108
BP_STEP_2D = 132
BN_STEP_2D = 108
BP_G2P_2D = 128
BN_G2P_2D = 28         # Δu read (2 floats) + m, p, f written (5 floats)


def advance_time(Ti, dt, n, f32):
    """Ti after n steps, accumulated as the library does (in FP32 for the
    reference's FP32 mode), so that the next call continues at the same time."""
    for _ in range(n):
        Ti = float(np.float32(np.float32(Ti) + np.float32(dt))) if f32 else Ti + dt
    return Ti


def fp64_device_rate(pkg, builder, published, device, K, W):
    """A reference example with every device array in FP64 (the precision of
    its published number): W untimed steps, then K steps timed with CUDA events."""
    case = getattr(pkg.workloads, builder)(gpu_precision="fp64")
    dev = pkg.DeviceModel(case.args, case.grid, case.mp, case.attr, case.bc, device=device)
    try:
        Ti = dev.step(case.dt, 0.0, W)
        dev.step_async(case.dt, Ti, K)
        dev.sync()
        ms = dev.stats().last_step_ms
    finally:
        dev.close()
    value = case.mp.np * K / (ms * 1e-3)
    return {"value": value, "unit": "particle-updates/s", "ms_per_step": ms / K,
            "vs_baseline": value / published}


def run_b200(args):
    rank, world, local = dist_env()
    pkg, case = make_case(args.mc3d, args.workload, args.surrogate)
    lib = pkg._lib
    use_dist = world > 1
    if use_dist:
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    npart = case.mp.np
    dt = case.dt
    K, W = args.steps, max(args.warmup, 3)

    # ---- end to end through the public API: host arrays -> device -> host ----
    pin_particles(case.mp)
    ts = getattr(case.mp, "phase", 1) == 2
    wkw = dict(phase=2, n=case.mp.n, rho_w=case.mp.rho_w) if ts else {}
    if case.grid.dim == 3:
        out = pkg.Particle3D(dx=case.mp.dx, dy=case.mp.dy, dz=case.mp.dz, xi=case.mp.xi, rho=case.mp.rho, **wkw)
    else:
        out = pkg.Particle2D(dx=case.mp.dx, dy=case.mp.dy, xi=case.mp.xi, rho=case.mp.rho, **wkw)
    pin_particles(out)
    ref_mask = lib.F_REFERENCE_TS if ts else lib.F_REFERENCE

    def e2e_once(nsteps):
        t0 = time.perf_counter()
        dev = pkg.DeviceModel(case.args, case.grid, case.mp, case.attr, case.bc, device=local)
        dev.step(dt, 0.0, nsteps)
        dev.download(ref_mask, out)
        t1 = time.perf_counter()
        dev.close()
        return t1 - t0

    # warm: context, module load, first allocations, and the first CUDA-graph
    # capture/instantiation (a block of two sort periods is replayed once a period has passed)
    e2e_once(max(W, 40))
    e2e_t = e2e_once(K)
    D = case.grid.dim
    nv = 6 if D == 3 else 4
    # uploaded particle columns (FP64: xi, vs, sig, eps, epsq/epsk/epsv, Omega/Omega0/rho/rho0, F) + nid
    h2d = npart * 8 * (D + D + nv + nv + 3 + 4 + D * D) + npart * 8
    # device2host! field set (FP64: sigm, vs, xi, Omega, sig, epsk, epsq, epsv, eps, ms)
    d2h = npart * 8 * (1 + D + D + 1 + nv + 1 + 1 + 1 + nv + 1)
    if ts:   # + n, ρw, σw, vw, ϵijw up; mw, vw, σw, ϵijw, n down
        h2d += npart * 8 * (3 + D + nv)
        d2h += npart * 8 * (3 + D + nv)

    # ---- device-timed region (inputs resident in HBM) ----
    dev = pkg.DeviceModel(case.args, case.grid, case.mp, case.attr, case.bc, device=local)
    tuning = None
    Ti = 0.0
    if args.workload == "batch2d":
        # untimed: the autotuner's trials are real steps of the model
        Ti, S, tiled, trial_ms = dev.autotune(dt, Ti, 16)
        tuning = {"sort_every": S, "variant": PASS_VARIANTS[tiled], "tile": dev.tile(), "trial_ms_per_step": trial_ms,
                  "candidates": "tile shapes x sort periods 8/16/32/64 (lane-merged passes), then the fused "
                                "pass at 3 CTAs/SM at 32/64, then tiled and box passes at 16/32 "
                                "(max(16, period) steps each), then the best variant-0 and the best "
                                "other candidate again back to back (64 steps each)"}
    surr_info = None
    if args.surrogate:
        if args.workload != "slope3d":
            raise SystemExit("--surrogate applies to --workload slope3d")
        # untimed: log samples of the plain return, train, switch the step over
        t0 = time.perf_counter()
        S = pkg.surrogate
        feat, tgt, Ti = S.collect_samples(dev, dt, Ti, 60, 6_000_000, every=8, device=local)
        sur = S.Surrogate(seed=1, device=local)
        sur.set_norm(feat, tgt)
        losses = sur.train(feat, tgt, epochs=6, batch=16384, lr=3e-3, lr_end=1e-4)
        # the plain step on the same state, for comparison
        Ti = dev.step(dt, Ti, 16)
        plain_ms = dev.stats().last_step_ms / 16
        dev.set_surrogate(sur, tol=1e-3, sref=1e3)
        surr_info = {"plain_ms_per_step_same_state": plain_ms,"train_samples": int(feat.shape[0]), "epochs": 6, "loss_first_last": [losses[0], losses[-1]],
                     "setup_s": time.perf_counter() - t0, "tol": 1e-3, "sref_pa": 1e3}
    Ti = dev.step(dt, Ti, W)
    if use_dist:
        dist.barrier()
    st0 = dev.stats()
    launches0, sorts0 = st0.launches, st0.sorts_done
    with ClockSampler(local) as clk:
        dev.step_async(dt, Ti, K)
        dev.sync()
    st = dev.stats()
    ms_window = st.last_step_ms
    launches = st.launches - launches0
    sorts_window = st.sorts_done - sorts0
    na = st.active_nodes
    Ti = advance_time(Ti, dt, K, dev.desc.time_f32)
    sort_used, tiled_used = dev.tuning()
    tile_used = dev.tile()
    if surr_info is not None:
        st_s = dev.stats()
        surr_info["rows"] = int(st_s.surr_rows)
        surr_info["accepted_fraction"] = 1.0 - st_s.surr_fallbacks / max(st_s.surr_rows, 1)

    # ---- per-kernel device times (events on the library stream), and the
    # cell re-sort, which runs every sort_used steps: the K-step window holds
    # whole sorts or none, so the reported time replaces the sorts it holds by
    # the amortised share sort_ms * K / sort_used ----
    dev.set_profiling(True)
    dev.step(dt, Ti, 16)
    for _ in range(3):
        dev.sort()
    kt = dev.kernel_times()
    dev.set_profiling(False)
    sort_ms = kt.get("sort", (0.0, 0))[0]
    ms = ms_window - sorts_window * sort_ms + sort_ms * K / sort_used
    t_max = max_over_ranks(ms, f"cuda:{local}") if use_dist else ms
    value = replica_value(world, npart, K, t_max)

    dev.close()
    dom = "g2p_p2g"
    dom_ms = kt.get(dom, (float("nan"), 0))[0]
    if dom not in kt and "g2p" in kt and "p2g" in kt:
        # surrogate steps run G2P and P2G as two passes around the MLP
        dom = "g2p+p2g"
        dom_ms = kt["g2p"][0] + kt["p2g"][0]
    elif dom not in kt and "g2p" in kt and "mvl_p2g" in kt:
        # MVL: G2P + update + cell sums, then the cell-averaged stress + P2G
        dom = "g2p+mvl_p2g"
        dom_ms = kt["g2p"][0] + kt["mvl_p2g"][0]
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    bp_g2p, bn_g2p = (BP_G2P_3D, BN_G2P_3D) if D == 3 else (BP_G2P_2D, BN_G2P_2D)
    bp_step, bn_step = (BP_STEP_3D, BN_STEP_3D) if D == 3 else (BP_STEP_2D, BN_STEP_2D)
    if args.workload == "saturated3d":
        bp_g2p, bn_g2p, bp_step, bn_step = BP_G2P_TS, BN_G2P_TS, BP_STEP_TS, BN_STEP_TS
    alg_bytes = npart * bp_g2p + na * bn_g2p
    achieved = alg_bytes / (dom_ms * 1e-3) / 1e9
    step_bytes = npart * bp_step + na * bn_step
    step_achieved = step_bytes / (ms * 1e-3 / K) / 1e9
    # DRAM bytes (read + write) per launch of the fused kernel, from one ncu
    # capture of this workload (--set full on k_g2p_chain), per particle
    traffic = G2P_TRAFFIC_PER_PARTICLE * npart if args.workload == "column3d" else None

    result = {
        "metric": "particle-updates/s", "value": value, "unit": "particle-updates/s",
        "n_gpus": world, "steps": K, "warmup": W, "ms_per_step": t_max / K,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.workload == "column2d" else "f32",
        "data": f"synthetic (seeded lattice + jitter, seed {case.meta['seed']})",
        "config": dict(WORKLOADS[args.workload],
                       particles=npart, nodes=case.grid.ni, active_nodes=na, h=case.meta["h"],
                       mc3d=args.mc3d, precision=("all FP64" if args.workload == "column2d"
                                                   else "FP32 bulk, FP64 positions and det(F)"), sort_every=sort_used,
                       particle_passes=PASS_VARIANTS[tiled_used], tile=tile_used,
                       l2=(f"particle state {npart * bp_step / 1e9:.2f} GB > 126 MB L2 (no flush needed)"
                           if npart * bp_step > 126e6 else
                           f"particle state {npart * bp_step / 1e6:.1f} MB < 126 MB L2: L2-resident, not "
                           "flushed (a model of this size runs from L2; launch-bound)"),
                       parallelism=f"replicas x{world}",
                       **({"tuning": tuning} if tuning else {}),
                       **({"slopes": len(case.meta["slopes"])} if "slopes" in case.meta else {}),
                       **({"surrogate": surr_info} if surr_info else {})),
        "gpu_launches": launches,
        "timed_window": {"ms_per_step": ms_window / K, "sorts": sorts_window, "sort_ms": sort_ms,
                         "sort_every": sort_used,
                         "note": "value and ms_per_step count the re-sort as sort_ms / sort_every per step"},
        "kernel_ms": {k: v[0] for k, v in kt.items()},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                     "peak_source": peak_src, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "alg_bytes_per_launch": alg_bytes,
                     "step_achieved": step_achieved, "step_frac": step_achieved / peak},
        "e2e": {"value": npart * K / e2e_t, "unit": "particle-updates/s",
                "h2d_bytes_per_step": h2d / K, "d2h_bytes_per_step": d2h / K, "steps": K,
                "what": "DeviceModel upload from pinned host arrays + K steps + device2host! field set"},
        "clocks": clk.summary(),
    }
    if args.workload in EXAMPLES:
        builder, published, source = EXAMPLES[args.workload]
        result["vs_baseline"] = value / published
        result["baseline"] = {"value": published, "unit": "particle-updates/s", "source": source}
        result["fp64_device"] = fp64_device_rate(pkg, builder, published, local, K, W)
    if args.snapshot_every > 0:
        result["snapshots"] = snapshot_cost(pkg, case, dt, K, args.snapshot_every, local)
    if args.workload == "column3d" and not args.no_extra:
        result["forms"] = extra_forms(pkg, local, K, W)
    if rank == 0 and not args.no_cpu_baseline:
        if args.workload in ("column3d", "column2d"):
            result["cpu_baseline"] = cpu_baseline(args.mc3d, args.workload)
    if use_dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(result))


def _timed_steps(dev, dt, Ti, K):
    """K steps timed on the device (CUDA events inside the library); returns
    (ms for the K steps, end time)."""
    dev.step_async(dt, Ti, K)
    dev.sync()
    ms = dev.stats().last_step_ms
    return ms, advance_time(Ti, dt, K, dev.desc.time_f32)


def extra_forms(pkg, local, K, W):
    """The batched and learned forms of the metric, beside the plain column:
    batch2d -- 256 independent 2D slopes in one grid (15.5 M particles),
    autotuned during untimed steps, K timed steps, and the run-out of two of
    its slopes against the same slopes stepped alone; slope3d -- the 8.0 M-
    particle 3D slope (lognormal cohesion field, Drucker-Prager) stepped
    plainly and with the trained stress-return surrogate from the same state
    (samples logged from 60 plain steps, 20 epochs of training on the device),
    with the surrogate's accepted fraction and its run-out / displacement
    error against the plain step after the same K steps."""
    out = {}
    # ---- batch2d ----
    case = pkg.workloads.slope_batch_2d(Te=0.0)
    dev = pkg.DeviceModel(case.args, case.grid, case.mp, case.attr, case.bc, device=local)
    try:
        Ti, S, tiled, trial_ms = dev.autotune(case.dt, 0.0, 16)
        n_pre = dev.stats().steps_done
        tile = dev.tile()
        Ti = dev.step(case.dt, Ti, W)
        ms, Ti = _timed_steps(dev, case.dt, Ti, K)
        xb = pkg.types.Particle2D(dx=case.mp.dx, dy=case.mp.dy, xi=case.mp.xi, rho=case.mp.rho)
        dev.download(pkg._lib.F_XI, xb)
    finally:
        dev.close()
    n_total = n_pre + W + K
    ro_b = pkg.workloads.slope_runouts(case, xb.xi)
    errs = []
    for k in (0, len(case.meta["slopes"]) // 2):
        single = pkg.workloads.slope_2d_single(case, k)
        d1 = pkg.DeviceModel(single.args, single.grid, single.mp, single.attr, single.bc, device=local)
        try:
            d1.step(single.dt, 0.0, n_total)
            x1 = pkg.types.Particle2D(dx=single.mp.dx, dy=single.mp.dy, xi=single.mp.xi, rho=single.mp.rho)
            d1.download(pkg._lib.F_XI, x1)
        finally:
            d1.close()
        ro_1 = pkg.workloads.slope_runouts(single, x1.xi)[0]
        errs.append(abs(ro_b[k] - ro_1) / max(abs(ro_1), case.meta["h"]))
    out["batch2d"] = {"workload": "256 independent 2D slopes in one grid (Drucker-Prager, FP32)",
                      "particles": int(case.mp.np), "ms_per_step": ms / K,
                      "particle_updates_per_s": case.mp.np * K / (ms * 1e-3),
                      "tuning": {"sort_every": S, "variant": PASS_VARIANTS[tiled], "tile": tile,
                                 "trial_ms_per_step": trial_ms},
                      "runout_err_vs_alone": {"slopes": 2, "steps": n_total, "max": max(errs)}}
    del case
    # ---- slope3d, plain and surrogate from the same state ----
    S_ = pkg.surrogate
    runs = {}
    for mode in ("plain", "surrogate"):
        case = pkg.workloads.slope_3d(Te=0.0)
        dev = pkg.DeviceModel(case.args, case.grid, case.mp, case.attr, case.bc, device=local)
        try:
            info = {}
            if mode == "surrogate":
                t0 = time.perf_counter()
                feat, tgt, Ti = S_.collect_samples(dev, case.dt, 0.0, 60, 6_000_000, every=8, device=local)
                sur = S_.Surrogate(seed=1, device=local)
                sur.set_norm(feat, tgt)
                losses = sur.train(feat, tgt, epochs=20, batch=16384, lr=3e-3, lr_end=1e-4)
                dev.set_surrogate(sur, tol=1e-3, sref=1e3)
                info = {"train_samples": int(feat.shape[0]), "epochs": 20,
                        "loss_first_last": [losses[0], losses[-1]], "setup_s": time.perf_counter() - t0}
                del feat, tgt
            else:
                Ti = dev.step(case.dt, 0.0, 60)
            Ti = dev.step(case.dt, Ti, W)
            ms, Ti = _timed_steps(dev, case.dt, Ti, K)
            st = dev.stats()
            x = pkg.types.Particle3D(dx=case.mp.dx, dy=case.mp.dy, dz=case.mp.dz, xi=case.mp.xi, rho=case.mp.rho)
            dev.download(pkg._lib.F_XI, x)
            if mode == "surrogate":
                info.update(rows=int(st.surr_rows),
                            accepted_fraction=1.0 - st.surr_fallbacks / max(st.surr_rows, 1))
            runs[mode] = (ms, x.xi.copy(), info, case.mp.xi.copy(), case.mp.np, case.meta["h"])
        finally:
            dev.close()
        del case
    ms_p, x_p, _, x0, npart, h = runs["plain"]
    ms_s, x_s, info, _, _, _ = runs["surrogate"]
    ro = lambda x: float(x[:, 0].max() - x0[:, 0].max())
    du_p, du_s = x_p - x0, x_s - x0
    info.update(ms_per_step=ms_s / K, particle_updates_per_s=npart * K / (ms_s * 1e-3),
                runout_err_vs_plain=abs(ro(x_s) - ro(x_p)) / max(abs(ro(x_p)), h),
                disp_rel_vs_plain=float(np.linalg.norm(du_s - du_p) / max(np.linalg.norm(du_p), 1e-300)))
    out["slope3d"] = {"workload": "3D slope, lognormal cohesion field, Drucker-Prager (plastic from the start)",
                      "particles": int(npart), "steps_compared": 60 + W + K,
                      "plain": {"ms_per_step": ms_p / K, "particle_updates_per_s": npart * K / (ms_p * 1e-3)},
                      "surrogate": info}
    return out


def snapshot_cost(pkg, case, dt, K, every, local):
    """Wall time of K steps in chunks of `every`, with and without a snapshot
    group (all nine fields, the model's float type) before each chunk; the
    snapshot's gather, copy and file write overlap the next chunk."""
    import shutil
    import tempfile
    T = np.float32 if case.args.precision == "FP32" else np.float64
    tmp = tempfile.mkdtemp(prefix="mpm_snap_")
    out = {"every": every, "steps": K}
    try:
        for mode in ("plain", "snapshots"):
            dev = pkg.DeviceModel(case.args, case.grid, case.mp, case.attr, case.bc, device=local)
            f = pkg.hdf5.H5File(os.path.join(tmp, "s.h5")) if mode == "snapshots" else None
            dev.step(dt, 0.0, 3)
            Ti, done, groups = 0.0, 0, 0
            t0 = time.perf_counter()
            while done < K:
                if f is not None:
                    groups += 1
                    dev.snapshot(f, groups, Ti, dtype=T)
                n = min(every, K - done)
                Ti = dev.step(dt, Ti, n)
                done += n
            if f is not None:
                dev.snapshot_wait()
                f.close()
            out[f"{mode}_ms_per_step"] = (time.perf_counter() - t0) * 1e3 / K
            dev.close()
            if f is not None:
                size = os.path.getsize(os.path.join(tmp, "s.h5"))
                out.update(groups=groups, file_bytes=size, bytes_per_group=size / groups)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    extra = out["snapshots_ms_per_step"] - out["plain_ms_per_step"]
    out["overhead_ms_per_group"] = extra * K / out["groups"]
    return out


def oracle_threads():
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()


def cpu_baseline(mc3d, workload="column3d", steps=None):
    """The FP64 CPU restatement of the reference path (OpenMP, all host cores)
    on the same workload: 1 warm-up step + a bounded number of timed steps
    (about 10 s of CPU work)."""
    from oracle import oracle as orc
    pkg, case = make_case(mc3d, workload)
    nth = oracle_threads()
    if steps is None:
        steps = max(2, min(4000, int(3e7 / case.mp.np)))
    o = orc.Oracle(case.args, case.grid, case.mp, case.attr, case.bc, nthreads=nth)
    o.run(case.dt, 0.0, 1)
    t0 = time.perf_counter()
    o.run(case.dt, case.dt, steps)
    t = time.perf_counter() - t0
    return {"value": case.mp.np * steps / t, "unit": "particle-updates/s", "cores": nth,
            "kind": "port", "sample": f"{steps} steps of the full {case.mp.np}-particle {workload} after 1 warm-up step"}


def run_reference(args):
    rank, world, local = dist_env()
    if rank != 0:
        return
    from oracle import oracle as orc
    pkg, case = make_case(args.mc3d)
    nth = oracle_threads()
    o = orc.Oracle(case.args, case.grid, case.mp, case.attr, case.bc, nthreads=nth)
    K, W = args.steps, max(args.warmup, 3)
    # each bench step: one MPM step of the full workload; bounded so the run ends in minutes
    t_first = time.perf_counter()
    o.run(case.dt, 0.0, 1)
    t1 = time.perf_counter() - t_first
    budget = 240.0
    Wr = min(W - 1, max(0, int(budget * 0.2 / max(t1, 1e-3))))
    o.run(case.dt, case.dt, Wr)
    Kr = K if (K * t1) < budget else max(1, int(budget / max(t1, 1e-3)))
    t0 = time.perf_counter()
    o.run(case.dt, (1 + Wr) * case.dt, Kr)
    t = time.perf_counter() - t0
    value = case.mp.np * Kr / t
    line = {
        "impl": "reference", "metric": "particle-updates/s", "value": value, "unit": "particle-updates/s",
        "n_gpus": world, "steps": K, "warmup": W, "ms_per_step": t / Kr * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seed 1002)",
        "config": {"workload": "3D granular column collapse, uGIMP, MUSL va=:a", "particles": case.mp.np,
                   "constitutive": "mohrcoulomb", "mc3d": args.mc3d,
                   "implementation": "FP64 C++ restatement of the reference CPU path (oracle/), OpenMP"},
        "cpu_baseline": {"value": value, "unit": "particle-updates/s", "cores": nth, "kind": "port",
                         "sample": f"{Kr} MPM steps of the full {case.mp.np}-particle column "
                                   f"(after {1 + Wr} warm-up steps)"},
        "e2e": {"value": value, "unit": "particle-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def run_profile(args):
    """Minimal launch sequence for profilers: upload, W + K steps, exit."""
    pkg, case = make_case(args.mc3d, args.workload)
    dev = pkg.DeviceModel(case.args, case.grid, case.mp, case.attr, case.bc)
    dev.step(case.dt, 0.0, args.warmup)
    dev.step(case.dt, args.warmup * case.dt, args.steps)
    st = dev.stats()
    dev.close()
    print(json.dumps({"profile_run": True, "steps": args.steps, "warmup": args.warmup,
                      "last_ms": st.last_step_ms, "launches": st.launches}))


def main():
    args = parse()
    if args.profile_run:
        run_profile(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
