"""The stress-return surrogate's tensor-core kernels (csrc/mpm_mlp.cu).

CPU: the parameter layout and normalisation helpers; the reference MLP's
backward against finite differences.  GPU: the tcgen05 forward against the
FP64 reference with the same BF16 roundings (tight) and without them (loose);
the tcgen05 gradient against the FP64 gradient; training lowers the loss.
"""
import numpy as np
import pytest

import mlp_ref
from helpers import rel


def rand_case(pkg, n, seed=0):
    S = pkg.surrogate
    rng = np.random.default_rng(seed)
    feat = rng.normal(0.0, 1.0, (n, 15)) * np.linspace(1.0, 3.0, 15) + np.linspace(-2.0, 2.0, 15)
    target = np.column_stack([np.tanh(feat[:, :6] * 0.5) + 0.1 * feat[:, 6:12] * feat[:, 12:13]])
    P = S.init_params(seed)
    norm = S.make_norm(feat, target)
    return S.pad_features(feat), target.astype(np.float32), P, norm


def test_param_layout(pkg):
    S = pkg.surrogate
    P = S.init_params(3)
    assert P.size == sum(k * n + n for k, n in S.LAYERS) == 10448
    layers = S.unpack(P)
    assert np.all(layers[0][0][15] == 0)          # padded input row
    assert np.all(layers[3][0][:, 6:] == 0)       # padded outputs
    assert all(np.all(b == 0) for _, b in layers)


def test_reference_gradient_matches_finite_differences(pkg):
    feat, target, P, norm = rand_case(pkg, 40, seed=1)
    layers = [(W.astype(np.float64), b.astype(np.float64) + 0.01) for W, b in pkg.surrogate.unpack(P)]
    grads, loss = mlp_ref.gradient(layers, norm, feat, target, 1.0 / 40)
    rng = np.random.default_rng(2)
    for li in range(4):
        W, b = layers[li]
        kmax = 15 if li == 0 else W.shape[0]
        nmax = 6 if li == 3 else W.shape[1]
        for _ in range(4):
            k, n = rng.integers(kmax), rng.integers(nmax)
            h = 1e-6
            Wp = W.copy(); Wp[k, n] += h
            Wm = W.copy(); Wm[k, n] -= h
            lp = mlp_ref.gradient(layers[:li] + [(Wp, b)] + layers[li + 1:], norm, feat, target, 1.0 / 40)[1]
            lm = mlp_ref.gradient(layers[:li] + [(Wm, b)] + layers[li + 1:], norm, feat, target, 1.0 / 40)[1]
            assert grads[li][0][k, n] == pytest.approx((lp - lm) / (2 * h), rel=1e-5, abs=1e-9)


def gpu_surrogate(pkg, P, norm):
    return pkg.surrogate.Surrogate(params=P, norm=norm, residual=False)


@pytest.mark.gpu
def test_forward_matches_reference(pkg, gpu_lib):
    import torch
    feat, target, P, norm = rand_case(pkg, 1000, seed=4)
    P = P.copy()
    for ow, ob in pkg.surrogate.offsets():   # nonzero biases
        P[ob:ob + 16] = np.linspace(-0.1, 0.1, 16, dtype=np.float32)
    layers = pkg.surrogate.unpack(P)
    layers[3][1][6:] = 0
    P[pkg.surrogate.offsets()[3][1] + 6:] = 0
    sur = gpu_surrogate(pkg, P, norm)
    out = sur.forward(torch.tensor(feat, device="cuda")).cpu().numpy()
    emu, _ = mlp_ref.forward(layers, norm, feat, emulate_bf16=True)
    exact, _ = mlp_ref.forward(layers, norm, feat, emulate_bf16=False)
    assert rel(out, emu) < 2e-3, rel(out, emu)
    assert rel(out, exact) < 3e-2, rel(out, exact)


@pytest.mark.gpu
def test_gradient_matches_reference(pkg, gpu_lib):
    import torch
    feat, target, P, norm = rand_case(pkg, 700, seed=5)   # 6 tiles, the last one partial
    layers = pkg.surrogate.unpack(P)
    sur = gpu_surrogate(pkg, P, norm)
    G, loss = sur.gradient(torch.tensor(feat, device="cuda"), torch.tensor(target, device="cuda"))
    ref, loss_ref = mlp_ref.gradient(layers, norm, feat, target, 1.0 / 700, emulate_bf16=True)
    ex, _ = mlp_ref.gradient(layers, norm, feat, target, 1.0 / 700, emulate_bf16=False)
    assert loss == pytest.approx(loss_ref, rel=2e-3)
    gl = pkg.surrogate.unpack(G)
    for li in range(4):
        assert rel(gl[li][0], ref[li][0]) < 1e-2, (li, rel(gl[li][0], ref[li][0]))
        assert rel(gl[li][1], ref[li][1]) < 1e-2, (li, rel(gl[li][1], ref[li][1]))
        assert rel(gl[li][0], ex[li][0]) < 4e-2, (li, rel(gl[li][0], ex[li][0]))


@pytest.mark.gpu
def test_training_lowers_the_loss(pkg, gpu_lib):
    import torch
    feat, target, P, norm = rand_case(pkg, 20000, seed=6)
    sur = gpu_surrogate(pkg, P, norm)
    losses = sur.train(torch.tensor(feat, device="cuda"), torch.tensor(target, device="cuda"), epochs=15,
                       batch=2048, lr=3e-3)
    assert losses[-1] < 0.1 * losses[0], losses


@pytest.mark.gpu
def test_residual_mode_adds_the_trial_stress(pkg, gpu_lib):
    """With the residual flag the network's output is the correction: the
    returned stress is trial + MLP, i.e. the plain output plus features 0..5."""
    import torch
    feat, target, P, norm = rand_case(pkg, 500, seed=7)
    a = pkg.surrogate.Surrogate(params=P, norm=norm, residual=False)
    b = pkg.surrogate.Surrogate(params=P, norm=norm, residual=True)
    x = torch.tensor(feat, device="cuda")
    oa = a.forward(x).cpu().numpy()
    ob = b.forward(x).cpu().numpy()
    assert np.allclose(ob, oa + feat[:, :6], rtol=1e-6, atol=1e-5 * np.abs(oa).max())


@pytest.mark.gpu
def test_completion_wait_timeout_is_reported(pkg, gpu_lib):
    """The bounded wait on the tensor-core completion barrier: with the test
    flag no MMA (and no commit) is issued, so the first wait runs out after
    its short limit; the kernel sets the error word and leaves with nothing in
    flight.  The host sees the error, and a normal call on the same context
    afterwards still succeeds and matches a fresh one."""
    import ctypes as C
    import torch
    feat, target, P, norm = rand_case(pkg, 300, seed=8)
    sur = gpu_surrogate(pkg, P, norm)
    x = torch.tensor(feat, device="cuda")
    good = sur.forward(x).cpu().numpy()
    out = torch.full((x.shape[0], 6), 7.0, device="cuda")
    sur.err.zero_()
    rc = gpu_lib.mpm_mlp_forward(sur.P.data_ptr(), sur.norm.data_ptr(), x.data_ptr(), out.data_ptr(),
                                 x.shape[0], sur.flags | 2, sur.err.data_ptr(),
                                 C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0
    torch.cuda.synchronize()
    assert int(sur.err.item()) & 1, "the timed-out wait was not reported"
    assert torch.all(out == 7.0), "a timed-out tile wrote output"
    with pytest.raises(pkg._lib.MPMError):
        sur._check_err()
    sur.err.zero_()
    again = sur.forward(x).cpu().numpy()
    torch.cuda.synchronize()
    assert int(sur.err.item()) == 0
    assert np.array_equal(again, good)
