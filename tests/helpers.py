"""Shared helpers for the parity tests."""
import numpy as np


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def fresh_particles(pkg, mp):
    """An output particle struct shaped like `mp` for downloads."""
    if mp.dim == 2:
        out = pkg.Particle2D(precision=mp.precision, dx=mp.dx, dy=mp.dy, xi=mp.xi, rho=mp.rho)
    else:
        out = pkg.Particle3D(precision=mp.precision, dx=mp.dx, dy=mp.dy, dz=mp.dz, xi=mp.xi, rho=mp.rho)
    return out
