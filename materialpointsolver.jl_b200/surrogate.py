"""The stress-return surrogate: a 15 -> 64 -> 64 -> 64 -> 6 GELU MLP, BF16
weights with FP32 accumulation, trained and run by the library's own
tensor-core kernels (csrc/mpm_mlp.cu, tcgen05).

No counterpart in the reference; it stands in for the Drucker-Prager return
(dpP!, src/materials/druckerprager.jl:89-155), which stays the fallback and the
judge of the network's error.  Features (15): trial stress (6, Voigt xx yy zz
xy yz zx), strain increment (6, engineering shear), accumulated plastic strain,
cohesion, friction angle (rad).  Output: the returned stress (6).

Device memory and streams come from torch (plumbing); every computation on
them is a kernel of libmpm_b200.so.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib

NF, NO, NFP = 15, 6, 16
LAYERS = [(16, 64), (64, 64), (64, 64), (64, 16)]   # padded (inputs, outputs)


def offsets():
    """(W offset, b offset) of each layer in the parameter vector."""
    out, o = [], 0
    for k, n in LAYERS:
        out.append((o, o + k * n))
        o += k * n + n
    return out


def init_params(seed=0):
    """Glorot-uniform weights on the real (unpadded) inputs / outputs, zero
    biases, zero padding."""
    rng = np.random.Generator(np.random.PCG64(seed))
    P = np.zeros(sum(k * n + n for k, n in LAYERS), np.float32)
    real = [(NF, 64), (64, 64), (64, 64), (64, NO)]
    for (ow, _), (k, n), (kr, nr) in zip(offsets(), LAYERS, real):
        lim = math.sqrt(6.0 / (kr + nr))
        W = np.zeros((k, n), np.float32)
        W[:kr, :nr] = rng.uniform(-lim, lim, size=(kr, nr))
        P[ow:ow + k * n] = W.ravel()
    return P


def unpack(P):
    """List of (W (k x n), b (n)) float arrays from a parameter vector."""
    P = np.asarray(P)
    return [(P[ow:ow + k * n].reshape(k, n), P[ob:ob + n]) for (ow, ob), (k, n) in zip(offsets(), LAYERS)]


def make_norm(feat, target, residual=False):
    """Per-column mean / std of features (15) and targets (6) -- of the
    correction target - trial stress when `residual` -- padded to the 64-float
    layout the kernels read; constant columns get std 1."""
    feat = np.asarray(feat, np.float64)
    target = np.asarray(target, np.float64)
    if residual:
        target = target - feat[:, :NO]
    norm = np.zeros(64, np.float32)
    fm, fs = feat[:, :NF].mean(0), feat[:, :NF].std(0)
    tm, ts = target.mean(0), target.std(0)
    fs[fs < 1e-12 * (1 + np.abs(fm))] = 1.0
    ts[ts < 1e-12 * (1 + np.abs(tm))] = 1.0
    norm[0:NF], norm[16:16 + NF] = fm, fs
    norm[16 + NF] = 1.0
    norm[32:32 + NO], norm[48:48 + NO] = tm, ts
    norm[48 + NO:64] = 1.0
    return norm


def pad_features(feat):
    """n x 15 -> n x 16 (FP32, zero pad column)."""
    feat = np.asarray(feat, np.float32)
    out = np.zeros((feat.shape[0], NFP), np.float32)
    out[:, :NF] = feat[:, :NF]
    return out


class Surrogate:
    """Parameters, normalisation and Adam state on one GPU."""

    def __init__(self, params=None, norm=None, device=0, seed=0, residual=True):
        import torch
        self.torch = torch
        # residual: the network predicts the plastic correction (returned minus
        # trial stress), which is small where the trial barely yields
        self.residual = bool(residual)
        self.flags = 1 if self.residual else 0
        self.dev = torch.device("cuda", device)
        L = _lib.lib()
        self.npar = L.mpm_mlp_nparams()
        P = init_params(seed) if params is None else np.asarray(params, np.float32)
        if P.size != self.npar:
            raise ValueError(f"expected {self.npar} parameters, got {P.size}")
        self.P = torch.tensor(P, device=self.dev)
        self.norm = torch.tensor(np.ones(64, np.float32) if norm is None else np.asarray(norm, np.float32),
                                 device=self.dev)
        if norm is None:
            self.norm[0:16] = 0
            self.norm[32:48] = 0
        self.G = torch.zeros(self.npar, device=self.dev)
        self.M = torch.zeros(self.npar, device=self.dev)
        self.V = torch.zeros(self.npar, device=self.dev)
        self.err = torch.zeros(1, dtype=torch.int32, device=self.dev)
        self.loss = torch.zeros(1, device=self.dev)
        self.steps = 0

    def _stream(self):
        return C.c_void_p(self.torch.cuda.current_stream(self.dev).cuda_stream)

    def _check_err(self):
        if int(self.err.item()) != 0:
            raise _lib.MPMError(-2, "tensor-core completion wait timed out in the surrogate kernels")

    def set_norm(self, feat, target):
        f = feat.cpu().numpy() if hasattr(feat, "cpu") else feat
        y = target.cpu().numpy() if hasattr(target, "cpu") else target
        self.norm.copy_(self.torch.tensor(make_norm(f, y, self.residual), device=self.dev))

    def forward(self, feat16):
        """feat16: n x 16 FP32 device tensor -> n x 6 FP32 device tensor."""
        t = self.torch
        feat16 = feat16.contiguous()
        n = feat16.shape[0]
        out = t.empty((n, NO), dtype=t.float32, device=self.dev)
        _lib.check(_lib.lib().mpm_mlp_forward(self.P.data_ptr(), self.norm.data_ptr(), feat16.data_ptr(),
                                              out.data_ptr(), n, self.flags, self.err.data_ptr(), self._stream()))
        return out

    def gradient(self, feat16, target, inv_btot=None):
        """Gradient (and loss) of the mean squared error in normalised units
        over the given samples, left in self.G / returned as numpy."""
        n = feat16.shape[0]
        self.G.zero_()
        self.loss.zero_()
        self._grad(feat16, target, 1.0 / n if inv_btot is None else inv_btot)
        self._check_err()
        return self.G.cpu().numpy(), float(self.loss.item())

    def _grad(self, feat16, target, inv_btot):
        _lib.check(_lib.lib().mpm_mlp_grad(self.P.data_ptr(), self.norm.data_ptr(), feat16.contiguous().data_ptr(),
                                           target.contiguous().data_ptr(), feat16.shape[0], float(inv_btot),
                                           self.flags, self.G.data_ptr(), self.loss.data_ptr(), self.err.data_ptr(),
                                           self._stream()))

    def train(self, feat16, target, epochs=10, batch=16384, lr=2e-3, seed=0, lr_end=None, log=None):
        """Adam on shuffled minibatches; returns the mean loss per epoch."""
        t = self.torch
        n = feat16.shape[0]
        g = t.Generator(device=self.dev)
        g.manual_seed(seed)
        losses = []
        nb = max(1, n // batch)
        total = epochs * nb
        for ep in range(epochs):
            perm = t.randperm(n, device=self.dev, generator=g)
            self.loss.zero_()
            for b in range(nb):
                idx = perm[b * batch:(b + 1) * batch]
                self.G.zero_()
                self._grad(feat16[idx], target[idx], 1.0 / idx.numel())
                self.steps += 1
                rate = lr if lr_end is None else lr * (lr_end / lr) ** (self.steps / total)
                _lib.check(_lib.lib().mpm_mlp_adam(self.P.data_ptr(), self.G.data_ptr(), self.M.data_ptr(),
                                                   self.V.data_ptr(), float(rate), 0.9, 0.999, 1e-8, self.steps,
                                                   self._stream()))
            losses.append(float(self.loss.item()) / nb)
            if log:
                log(ep, losses[-1])
        self._check_err()
        return losses

    def params(self):
        return self.P.cpu().numpy()


def collect_samples(dev, dt, Ti, nsteps, cap, every=1, device=0):
    """Run `nsteps` plain steps of a DeviceModel from time Ti while logging
    training samples of the Drucker-Prager return; returns (features n x 16,
    targets n x 6 as device tensors, end time)."""
    import torch
    d = torch.device("cuda", device)
    feat = torch.zeros((cap, NFP), dtype=torch.float32, device=d)
    tgt = torch.zeros((cap, NO), dtype=torch.float32, device=d)
    cnt = torch.zeros(1, dtype=torch.int32, device=d)
    dev.log_samples(feat, tgt, cnt, every)
    try:
        Ti = dev.step(dt, Ti, nsteps)
    finally:
        dev.log_samples(None, None, None, 0)
    n = min(int(cnt.item()) & 0xFFFFFFFF, cap)
    return feat[:n], tgt[:n], Ti


FLOP_FORWARD = 2 * (NF * 64 + 64 * 64 + 64 * 64 + 64 * NO)   # 19 072 per sample (unpadded)
