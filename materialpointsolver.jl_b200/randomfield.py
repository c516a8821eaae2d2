"""Gaussian random fields by the randomised spectral method (Räss, Kolyukhin &
Minakov 2019), the host side of grf_gc! / grf_ec!
(src/toolkits/randomfield.jl:57-96, 112-150).

The harmonics are drawn on the host with numpy's PCG64 following the
reference's sampling steps (its Julia rand/randn stream cannot be reproduced);
the O(np x Nh) sum runs on the GPU through ``mpm_grf_eval``.

``rescale="minmax"`` maps the field onto [rl, rr] like the reference.
``rescale="standard"`` instead standardises it to zero mean and unit variance,
which is what a lognormal material field needs (``lognormal``).
"""
from __future__ import annotations

import math

import numpy as np

from . import _lib


def harmonics_gc(rng, If=2.0, k_m=100.0, Nh=5000):
    """Harmonics of the Gaussian-covariance field, randomfield.jl:72-88: random
    phase, a wavenumber drawn by rejection from k^2 exp(-k^2/2) on [0, k_m)
    scaled by sqrt(2)/lf with lf = 1.128379 If, an isotropic direction, and
    N(0, 1) amplitudes.  Returns an (Nh, 5) array of (V1, V2, V3, a, b)."""
    H = np.empty((Nh, 5))
    lf = 1.128379 * If
    for j in range(Nh):
        fi = 6.283185 * rng.random()
        while True:
            k = k_m * rng.random()
            d = k * k * math.exp(-0.5 * k * k)
            if not rng.random() * 0.735759 >= d:
                break
        k = 1.414214 * k / lf
        theta = math.acos(1.0 - 2.0 * rng.random())
        H[j, 0] = k * math.sin(fi) * math.sin(theta)
        H[j, 1] = k * math.cos(fi) * math.sin(theta)
        H[j, 2] = k * math.cos(theta)
        H[j, 3] = rng.standard_normal()
        H[j, 4] = rng.standard_normal()
    return H


def harmonics_ec(rng, If=(10.0, 8.0, 5.0), Nh=5000):
    """Harmonics of the exponential-covariance field, randomfield.jl:127-143:
    k = tan(pi/2 u) accepted with probability k^2 / (1 + k^2), anisotropic
    correlation lengths If = (x, y, z)."""
    H = np.empty((Nh, 5))
    for j in range(Nh):
        fi = 6.283185 * rng.random()
        while True:
            k = math.tan(1.570796 * rng.random())
            d = (k * k) / (1.0 + k * k)
            if rng.random() < d:
                break
        theta = math.acos(1.0 - 2.0 * rng.random())
        H[j, 0] = k * math.sin(fi) * math.sin(theta) / If[0]
        H[j, 1] = k * math.cos(fi) * math.sin(theta) / If[1]
        H[j, 2] = k * math.cos(theta) / If[2]
        H[j, 3] = rng.standard_normal()
        H[j, 4] = rng.standard_normal()
    return H


def evaluate(pts, H, scale, device=0):
    """scale * sum_j (a_j sin(V_j.p) + b_j cos(V_j.p)) at every row of pts (np x 2
    or np x 3), on the GPU in FP64."""
    pts = np.asarray(pts, dtype=np.float64)
    npts = pts.shape[0]
    cols = [np.ascontiguousarray(pts[:, d]) for d in range(pts.shape[1])]
    z = cols[2] if len(cols) > 2 else None
    H = np.ascontiguousarray(H, dtype=np.float64)
    out = np.empty(npts)
    L = _lib.lib()
    rc = L.mpm_grf_eval(device, cols[0].ctypes.data, cols[1].ctypes.data, z.ctypes.data if z is not None else None,
                        npts, H.ctypes.data, H.shape[0], float(scale), out.ctypes.data)
    _lib.check(rc)
    return out


def _finish(Y, rl, rr, rescale):
    if rescale == "minmax":
        lo, hi = min(rl, rr), max(rl, rr)
        mx, mn = Y.max(), Y.min()
        return (Y - mn) / (mx - mn) * (hi - lo) + lo
    if rescale == "standard":
        return (Y - Y.mean()) / Y.std()
    if rescale is None:
        return Y
    raise ValueError(f"unknown rescale {rescale!r}")


def grf_gc(Yf, pts, rl, rr, *, If=2.0, k_m=100.0, Nh=5000, sf=1.0, seed=0, rescale="minmax", device=0):
    """grf_gc!(Yf, pts, rl, rr; If, k_m, Nh, sf): Gaussian covariance with
    correlation length If.  Fills and returns Yf."""
    H = harmonics_gc(np.random.Generator(np.random.PCG64(seed)), If=If, k_m=k_m, Nh=Nh)
    Y = evaluate(pts, H, sf / math.sqrt(Nh), device)
    Yf[:] = _finish(Y, rl, rr, rescale)
    return Yf


def grf_ec(Yf, pts, rl, rr, *, If=(10.0, 8.0, 5.0), Nh=5000, sf=1.0, seed=0, rescale="minmax", device=0):
    """grf_ec!(Yf, pts, rl, rr; If, Nh, sf): exponential covariance with
    per-axis correlation lengths If.  Fills and returns Yf."""
    H = harmonics_ec(np.random.Generator(np.random.PCG64(seed)), If=If, Nh=Nh)
    Y = evaluate(pts, H, sf / math.sqrt(Nh), device)
    Yf[:] = _finish(Y, rl, rr, rescale)
    return Yf


def lognormal(Z, mean, cov):
    """Lognormal values with the given mean and coefficient of variation from a
    standard normal field Z: sigma_ln^2 = ln(1 + cov^2), mu_ln = ln(mean) -
    sigma_ln^2 / 2."""
    s2 = math.log(1.0 + cov * cov)
    mu = math.log(mean) - 0.5 * s2
    return np.exp(mu + math.sqrt(s2) * np.asarray(Z))
