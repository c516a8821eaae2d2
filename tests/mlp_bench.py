"""Timing of the surrogate MLP's tensor-core forward and gradient kernels on
random samples (a measurement driver, not part of the library).

Run:  python tests/mlp_bench.py [n]
"""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def benchmark(n=2_000_000, reps=20, device=0):
    """Time the tensor-core forward and gradient kernels on n random samples;
    prints and returns samples/s and TFLOP/s (unpadded FLOP count; the
    backward counts twice the forward)."""
    import __graft_entry__ as g
    S = g.load_package().surrogate
    Surrogate, NF, NFP, NO, FLOP_FORWARD = S.Surrogate, S.NF, S.NFP, S.NO, S.FLOP_FORWARD
    import json
    import torch
    d = torch.device("cuda", device)
    g = torch.Generator(device=d)
    g.manual_seed(0)
    feat = torch.randn((n, NFP), generator=g, device=d)
    feat[:, NF] = 0
    tgt = torch.randn((n, NO), generator=g, device=d)
    sur = Surrogate(seed=0, device=device, residual=False)
    sur.set_norm(feat[:4096].cpu().numpy(), tgt[:4096].cpu().numpy())
    for _ in range(3):
        sur.forward(feat)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        sur.forward(feat)
    e1.record()
    torch.cuda.synchronize()
    fwd_ms = e0.elapsed_time(e1) / reps
    sur._grad(feat, tgt, 1.0 / n)
    e0.record()
    for _ in range(reps):
        sur._grad(feat, tgt, 1.0 / n)
    e1.record()
    torch.cuda.synchronize()
    grad_ms = e0.elapsed_time(e1) / reps
    sur._check_err()
    out = {"samples": n, "forward_ms": fwd_ms, "forward_samples_per_s": n / (fwd_ms * 1e-3),
           "forward_tflops": n * FLOP_FORWARD / (fwd_ms * 1e-3) / 1e12,
           "grad_ms": grad_ms, "grad_tflops": 3 * n * FLOP_FORWARD / (grad_ms * 1e-3) / 1e12}
    print(json.dumps(out))
    return out


if __name__ == "__main__":
    benchmark(int(sys.argv[1]) if len(sys.argv) > 1 else 2_000_000)
