"""CPU reference of the surrogate MLP (test infrastructure): forward and
backward in FP64, optionally rounding to BF16 at exactly the points where the
tensor-core kernels hold BF16 operands (normalised inputs, weights, hidden
activations, back-propagated pre-activation gradients)."""
import math

import numpy as np


def bf16(x):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    a = np.ascontiguousarray(np.asarray(x, np.float32)).view(np.uint32)
    r = ((a + np.uint32(0x7FFF) + ((a >> np.uint32(16)) & np.uint32(1))) & np.uint32(0xFFFF0000)).view(np.float32)
    return r.astype(np.float64)


GELU_K, GELU_A = math.sqrt(2.0 / math.pi), 0.044715


def gelu(z):
    """GELU, tanh form (Hendrycks & Gimpel 2016), as the device kernels use."""
    return 0.5 * z * (1.0 + np.tanh(GELU_K * (z + GELU_A * z ** 3)))


def gelu_grad(z):
    t = np.tanh(GELU_K * (z + GELU_A * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * GELU_K * (1.0 + 3.0 * GELU_A * z * z)


def forward(layers, norm, feat16, emulate_bf16=False):
    """layers: [(W k x n, b n)], norm: 64 floats, feat16: n x 16.  Returns
    (outputs in physical units n x 6, cache for backward)."""
    r = bf16 if emulate_bf16 else (lambda v: np.asarray(v, np.float64))
    norm = np.asarray(norm, np.float64)
    x = (np.asarray(feat16, np.float64)[:, :15] - norm[:15]) / norm[16:31]
    x = np.column_stack([x, np.zeros(len(x))])
    a = r(x)
    cache = [a]
    zs = []
    for li, (W, b) in enumerate(layers):
        z = a @ r(W) + np.asarray(b, np.float64)
        zs.append(z)
        if li < 3:
            a = r(gelu(z))
            cache.append(a)
    out = zs[-1][:, :6] * norm[48:54] + norm[32:38]
    return out, (cache, zs)


def gradient(layers, norm, feat16, target, inv_btot, emulate_bf16=False):
    """Gradient of 1/2 * inv_btot * sum (yhat - y)^2 (normalised units) with
    respect to every (W, b); returns ([(dW, db)], loss)."""
    r = bf16 if emulate_bf16 else (lambda v: np.asarray(v, np.float64))
    norm = np.asarray(norm, np.float64)
    _, (acts, zs) = forward(layers, norm, feat16, emulate_bf16)
    y = (np.asarray(target, np.float64) - norm[32:38]) / norm[48:54]
    d = np.zeros_like(zs[-1])
    d[:, :6] = zs[-1][:, :6] - y
    loss = 0.5 * inv_btot * float((d[:, :6] ** 2).sum())
    d *= inv_btot
    grads = [None] * 4
    for li in range(3, -1, -1):
        W, _ = layers[li]
        dz = r(d)
        grads[li] = (acts[li].T @ dz, d.sum(0))
        if li > 0:
            dy = dz @ r(W).T
            d = dy * gelu_grad(zs[li - 1])
    return grads, loss
