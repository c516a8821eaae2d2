"""Shared helpers for the parity tests."""
import numpy as np


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def fresh_particles(pkg, mp):
    """An output particle struct shaped like `mp` for downloads."""
    w = dict(phase=2, n=mp.n, rho_w=mp.rho_w) if getattr(mp, "phase", 1) == 2 else {}
    if mp.dim == 2:
        out = pkg.Particle2D(precision=mp.precision, dx=mp.dx, dy=mp.dy, xi=mp.xi, rho=mp.rho, **w)
    else:
        out = pkg.Particle3D(precision=mp.precision, dx=mp.dx, dy=mp.dy, dz=mp.dz, xi=mp.xi, rho=mp.rho, **w)
    return out
