"""Seeded synthetic inputs for the benchmark configurations.

The reference publishes no dataset for this path; these builders produce the
granular column-collapse and slope inputs with the sizes, material constants
and boundary conditions the configurations name, through the same host
constructors a reference user calls (UserArgs*, UserGrid*, UserParticle*,
UserProperty, UserVBoundary*).  Positions are a regular lattice of lp = h/2
(2 particles per cell per axis) with a seeded uniform jitter.
"""
from __future__ import annotations

import math

import numpy as np

from .types import (UserArgs2D, UserArgs3D, UserGrid2D, UserGrid3D, UserParticle2D,
                    UserParticle3D, UserProperty, UserVBoundary2D, UserVBoundary3D,
                    jl_range, meshbuilder)


def elastic_constants(E, nu):
    K = E / (3.0 * (1.0 - 2.0 * nu))
    G = E / (2.0 * (1.0 + nu))
    return K, G


def cfl_dt(h, K, G, rho, cfl=0.2):
    """Δt = CFL·h / c_p with the P-wave speed c_p = sqrt((K + 4G/3)/ρ)."""
    return cfl * h / math.sqrt((K + 4.0 * G / 3.0) / rho)


class Case:
    """A ready-to-run set of reference-style structs plus run metadata."""

    def __init__(self, name, args, grid, mp, attr, bc, dt, nsteps_full, meta):
        self.name, self.args, self.grid, self.mp, self.attr, self.bc = name, args, grid, mp, attr, bc
        self.dt = dt
        self.nsteps_full = nsteps_full
        self.meta = meta


def column_collapse_2d(*, h=0.005, ppc=2, seed=1001, jitter=0.1, width=0.2, height=0.1,
                       domain=(0.6, 0.15), pad=2, precision="FP64", constitutive="druckerprager",
                       E=0.84e6, nu=0.3, rho=2650.0, phi_deg=19.8, c=0.0, psi_deg=0.0,
                       gravity=-9.81, Ttol=1.0, cfl=0.2, gpu_precision="mixed", project_path="/tmp",
                       **extra):
    """2D granular column collapse (uGIMP, plane strain).  Defaults: domain
    0.6 x 0.15 m, h = 5 mm, 2x2 particles per cell in a 0.2 x 0.1 m column
    (3 200 particles), DP with friction 19.8°, cohesion 0, dilation 0, fixed
    left wall, free-slip floor, CFL 0.2, 1 s.  The grid carries `pad` extra
    cells on every side so no particle's stencil leaves it."""
    K, G = elastic_constants(E, nu)
    dt = cfl_dt(h, K, G, rho, cfl)
    lp = h / ppc
    rng = np.random.Generator(np.random.PCG64(seed))
    xs = jl_range(lp / 2, lp, width - lp / 2)
    ys = jl_range(lp / 2, lp, height - lp / 2)
    pts = meshbuilder(xs, ys)
    pts = pts + rng.uniform(-jitter * h, jitter * h, size=pts.shape)
    npart = pts.shape[0]
    akw = dict(Ttol=Ttol, Te=0, ΔT=dt, FLIP=1, PIC=0, constitutive=constitutive, basis="uGIMP",
               device="B200", coupling="OS", scheme="MUSL", va="a", gravity=gravity, ζs=0,
               project_name="column2d", project_path=project_path, ϵ=precision,
               gpu_precision=gpu_precision, make_project_dir=False)
    akw.update(extra)
    args = UserArgs2D(**akw)
    grid = UserGrid2D(ϵ=precision, x1=-pad * h, x2=domain[0] + pad * h, y1=-pad * h,
                      y2=domain[1] + pad * h, dx=h, dy=h, NIC=9)
    mp = UserParticle2D(ϵ=precision, NIC=9, dx=lp, dy=lp, ξ=pts, ρs=np.full(npart, rho))
    attr = UserProperty(ϵ=precision, nid=np.ones(npart, np.int64), ν=[nu], Es=[E], Gs=[G], Ks=[K],
                        σt=[0.0], ϕ=[math.radians(phi_deg)], ϕr=[0.0], ψ=[math.radians(psi_deg)],
                        c=[c], cr=[0.0], Hp=[0.0])
    gx = grid.xi[:, 0]
    gy = grid.xi[:, 1]
    eps = 1e-9 * h
    left = gx <= 0.0 + eps
    right = gx >= domain[0] - eps
    floor = gy <= 0.0 + eps
    vx_idx = (left | right).astype(np.int64)
    vy_idx = (left | floor).astype(np.int64)
    bc = UserVBoundary2D(ϵ=precision, vx_s_idx=vx_idx, vx_s_val=np.zeros(grid.ni),
                         vy_s_idx=vy_idx, vy_s_val=np.zeros(grid.ni))
    nsteps = int(math.ceil(Ttol / dt))
    return Case("column_collapse_2d", args, grid, mp, attr, bc, dt, nsteps,
                dict(np=npart, h=h, K=K, G=G, seed=seed))


def column_collapse_3d(*, h=0.005, ppc=2, seed=1002, jitter=0.1, column=(0.5, 0.2, 0.4),
                       domain=(1.2, 0.4, 0.6), pad=2, precision="FP64", constitutive="mohrcoulomb",
                       E=1.0e6, nu=0.3, rho=2650.0, phi_deg=30.0, c=0.0, psi_deg=0.0, gravity=-9.81,
                       Ttol=1.0, cfl=0.2, gpu_precision="mixed", mc3d="literal", project_path="/tmp", sigt=0.0,
                       **extra):
    """3D granular column collapse.  Defaults: domain 1.2 x 0.4 x 0.6 m
    (z up), h = 5 mm, 2x2x2 particles per cell in a 0.5 x 0.2 x 0.4 m column
    (2 560 000 particles), Mohr-Coulomb φ = 30°, c = 0, ψ = 0, ρ = 2650,
    E = 1 MPa, ν = 0.3, free-slip walls and floor, CFL 0.2, 1 s."""
    K, G = elastic_constants(E, nu)
    dt = cfl_dt(h, K, G, rho, cfl)
    lp = h / ppc
    rng = np.random.Generator(np.random.PCG64(seed))
    xs = jl_range(lp / 2, lp, column[0] - lp / 2)
    ys = jl_range(lp / 2, lp, column[1] - lp / 2)
    zs = jl_range(lp / 2, lp, column[2] - lp / 2)
    pts = meshbuilder(xs, ys, zs)
    pts += rng.uniform(-jitter * h, jitter * h, size=pts.shape)
    npart = pts.shape[0]
    akw = dict(Ttol=Ttol, Te=0, ΔT=dt, FLIP=1, PIC=0, constitutive=constitutive, basis="uGIMP",
               device="B200", coupling="OS", scheme="MUSL", va="a", gravity=gravity, ζs=0,
               project_name="column3d", project_path=project_path, ϵ=precision,
               gpu_precision=gpu_precision, mc3d=mc3d, make_project_dir=False)
    akw.update(extra)
    args = UserArgs3D(**akw)
    grid = UserGrid3D(ϵ=precision, x1=-pad * h, x2=domain[0] + pad * h, y1=-pad * h,
                      y2=domain[1] + pad * h, z1=-pad * h, z2=domain[2] + pad * h, dx=h, dy=h, dz=h,
                      NIC=27)
    mp = UserParticle3D(ϵ=precision, NIC=27, dx=lp, dy=lp, dz=lp, ξ=pts, ρs=np.full(npart, rho))
    attr = UserProperty(ϵ=precision, nid=np.ones(npart, np.int64), ν=[nu], Es=[E], Gs=[G], Ks=[K],
                        σt=[sigt], ϕ=[math.radians(phi_deg)], ϕr=[0.0], ψ=[math.radians(psi_deg)],
                        c=[c], cr=[0.0], Hp=[0.0])
    # boundary flags per node, built from the node coordinates without forming grid.ξ
    nnx, nny, nnz = grid.nnx, grid.nny, grid.nnz
    vx = grid._vx
    vy = grid._vy
    vz = grid._vz
    eps = 1e-9 * h
    bx = ((vx <= eps) | (vx >= domain[0] - eps))
    by = ((vy <= eps) | (vy >= domain[1] - eps))
    bz = (vz <= eps)
    # node id = (iz*nnx + ix)*nny + iy
    fx = np.broadcast_to(bx[None, :, None], (nnz, nnx, nny)).ravel().astype(np.int64)
    fy = np.broadcast_to(by[None, None, :], (nnz, nnx, nny)).ravel().astype(np.int64)
    fz = np.broadcast_to(bz[:, None, None], (nnz, nnx, nny)).ravel().astype(np.int64)
    zeros = np.zeros(grid.ni)
    bc = UserVBoundary3D(ϵ=precision, vx_s_idx=fx, vx_s_val=zeros, vy_s_idx=fy, vy_s_val=zeros,
                         vz_s_idx=fz, vz_s_val=zeros)
    nsteps = int(math.ceil(Ttol / dt))
    return Case("column_collapse_3d", args, grid, mp, attr, bc, dt, nsteps,
                dict(np=npart, h=h, K=K, G=G, seed=seed))


def small_column_3d(**kw):
    """A scaled-down 3D column (same physics and boundary conditions) that the
    oracle steps in well under a second."""
    base = dict(h=0.02, column=(0.2, 0.1, 0.16), domain=(0.4, 0.16, 0.24), seed=1002)
    base.update(kw)
    return column_collapse_3d(**base)


def slope_points_3d(h, ppc, height, crest, slope_deg, width, rng, jitter=0.1):
    """Lattice particles (lp = h/ppc, seeded jitter) filling a slope of the given
    height against the x = 0 wall: a crest of length `crest`, then a face at
    `slope_deg` down to the toe, over the full width in y (z up)."""
    lp = h / ppc
    tb = math.tan(math.radians(slope_deg))
    x_toe = crest + height / tb
    xs = jl_range(lp / 2, lp, x_toe - lp / 2)
    ys = jl_range(lp / 2, lp, width - lp / 2)
    zs = jl_range(lp / 2, lp, height - lp / 2)
    pts = meshbuilder(xs, ys, zs)
    keep = pts[:, 0] <= crest + (height - pts[:, 2]) / tb
    pts = pts[keep]
    pts += rng.uniform(-jitter * h, jitter * h, size=pts.shape)
    return pts


def slope_3d(*, h=0.1, ppc=2, seed=1003, jitter=0.1, domain=(100.0, 20.0, 40.0), height=6.0, crest=4.05,
             slope_deg=35.0, pad=2, precision="FP64", E=20.0e6, nu=0.3, rho=2000.0, phi_deg=25.0, psi_deg=0.0,
             c_mean=10.0e3, c_cov=0.3, corr_len=2.0, nh=5000, k_m=100.0, field=True, gravity=-9.81,
             Ttol=10.0, Te=1.0, cfl=0.2, gpu_precision="mixed", project_path="/tmp", device=0, **extra):
    """3D slope failure: a 35° slope of height 6 m and crest 4.05 m against the
    x = 0 wall, 20 m wide, in a 100 x 20 x 40 m domain at h = 0.1 m with 2x2x2
    particles per cell (8 000 particles per m^3): 50 m^2 x 20 m = 1 000 m^3, so
    about 8.0 M particles.  Drucker-Prager φ = 25°, ψ = 0, E = 20 MPa, ν = 0.3,
    ρ = 2000, gravity ramped over Te = 1 s, 10 s simulated.  Cohesion is a
    lognormal random field (mean 10 kPa, CoV 0.3) over a Gaussian-covariance
    field of correlation length 2 m (grf_gc's randomised spectral method with
    5 000 harmonics, standardised to N(0, 1)), one material per particle like
    the reference expresses a random field (nid = 1:np).  field=False gives the
    uniform mean cohesion instead.  Boundaries: floor fixed, x and y walls
    free-slip."""
    from . import randomfield
    K, G = elastic_constants(E, nu)
    dt = cfl_dt(h, K, G, rho, cfl)
    lp = h / ppc
    rng = np.random.Generator(np.random.PCG64(seed))
    pts = slope_points_3d(h, ppc, height, crest, slope_deg, domain[1], rng, jitter)
    npart = pts.shape[0]
    if field:
        Z = randomfield.grf_gc(np.empty(npart), pts, 0.0, 1.0, If=corr_len, k_m=k_m, Nh=nh, seed=seed,
                               rescale="standard", device=device)
        coh = randomfield.lognormal(Z, c_mean, c_cov)
        nid = np.arange(1, npart + 1, dtype=np.int64)
    else:
        coh = np.array([c_mean])
        nid = np.ones(npart, np.int64)
    nm = coh.shape[0]

    def full(v):
        return np.full(nm, v, dtype=np.float64)

    akw = dict(Ttol=Ttol, Te=Te, ΔT=dt, FLIP=1, PIC=0, constitutive="druckerprager", basis="uGIMP",
               device="B200", coupling="OS", scheme="MUSL", va="a", gravity=gravity, ζs=0,
               project_name="slope3d", project_path=project_path, ϵ=precision, gpu_precision=gpu_precision,
               make_project_dir=False)
    akw.update(extra)
    args = UserArgs3D(**akw)
    grid = UserGrid3D(ϵ=precision, x1=-pad * h, x2=domain[0] + pad * h, y1=-pad * h, y2=domain[1] + pad * h,
                      z1=-pad * h, z2=domain[2] + pad * h, dx=h, dy=h, dz=h, NIC=27)
    mp = UserParticle3D(ϵ=precision, NIC=27, dx=lp, dy=lp, dz=lp, ξ=pts, ρs=np.full(npart, rho))
    attr = UserProperty(ϵ=precision, nid=nid, ν=full(nu), Es=full(E), Gs=full(G), Ks=full(K), σt=full(0.0),
                        ϕ=full(math.radians(phi_deg)), ϕr=full(0.0), ψ=full(math.radians(psi_deg)), c=coh,
                        cr=full(0.0), Hp=full(0.0))
    nnx, nny, nnz = grid.nnx, grid.nny, grid.nnz
    eps = 1e-9 * h
    vx, vy, vz = grid._vx, grid._vy, grid._vz
    bx = ((vx <= eps) | (vx >= domain[0] - eps))
    by = ((vy <= eps) | (vy >= domain[1] - eps))
    bz = (vz <= eps)
    fx = np.broadcast_to(bx[None, :, None] | bz[:, None, None], (nnz, nnx, nny)).ravel().astype(np.int64)
    fy = np.broadcast_to(by[None, None, :] | bz[:, None, None], (nnz, nnx, nny)).ravel().astype(np.int64)
    fz = np.broadcast_to(bz[:, None, None], (nnz, nnx, nny)).ravel().astype(np.int64)
    zeros = np.zeros(grid.ni)
    bc = UserVBoundary3D(ϵ=precision, vx_s_idx=fx, vx_s_val=zeros, vy_s_idx=fy, vy_s_val=zeros,
                         vz_s_idx=fz, vz_s_val=zeros)
    nsteps = int(math.ceil(Ttol / dt))
    return Case("slope_3d", args, grid, mp, attr, bc, dt, nsteps,
                dict(np=npart, h=h, K=K, G=G, seed=seed, cohesion=coh if field else None))


# ---------------------------------------------------------------------------
# Batches of independent 2D slopes packed side by side into one grid
# ---------------------------------------------------------------------------
def draw_slope_specs(n, seed=1004, np_range=(1.0e4, 2.0e5), angle_deg=(25.0, 45.0), height=(5.0, 20.0),
                     cohesion=(0.0, 20.0e3), friction_deg=(20.0, 35.0), h=0.05, ppc=2):
    """Draw n slopes: particle count log-uniform in np_range, angle, height,
    cohesion and friction uniform.  The cross-section area that holds the drawn
    count is a triangle of the drawn height and angle plus a crest; when the
    triangle alone is already larger, the height is lowered instead (same
    angle, no crest)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    per_area = (ppc / h) ** 2
    specs = []
    for s in range(n):
        target = float(np.exp(rng.uniform(math.log(np_range[0]), math.log(np_range[1]))))
        beta = math.radians(rng.uniform(*angle_deg))
        H = rng.uniform(*height)
        c = rng.uniform(*cohesion)
        phi = math.radians(rng.uniform(*friction_deg))
        area = target / per_area
        tri = H * H / (2.0 * math.tan(beta))
        if area >= tri:
            crest = (area - tri) / H
        else:
            H = math.sqrt(2.0 * area * math.tan(beta))
            crest = 0.0
        specs.append(dict(index=s, target_np=target, beta=beta, H=H, crest=crest, c=c, phi=phi,
                          seed=int(rng.integers(1 << 62))))
    return specs


def slope_points_2d(spec, h, ppc=2, jitter=0.1):
    """Lattice particles of one slope in its local frame (left wall x = 0, floor
    y = 0), with the slope's own seeded jitter."""
    lp = h / ppc
    tb = math.tan(spec["beta"])
    x_toe = spec["crest"] + spec["H"] / tb
    xs = jl_range(lp / 2, lp, x_toe - lp / 2)
    ys = jl_range(lp / 2, lp, spec["H"] - lp / 2)
    pts = meshbuilder(xs, ys)
    pts = pts[pts[:, 0] <= spec["crest"] + (spec["H"] - pts[:, 1]) / tb]
    rng = np.random.Generator(np.random.PCG64(spec["seed"]))
    return pts + rng.uniform(-jitter * h, jitter * h, size=pts.shape)


def slope_batch_2d(*, n_slopes=256, seed=1004, specs=None, h=0.05, ppc=2, jitter=0.1, gap_cells=8, pad=2,
                   runout_factor=3.0, precision="FP64", E=20.0e6, nu=0.3, rho=2000.0, psi_deg=0.0, gravity=-9.81,
                   Ttol=5.0, Te=0.5, cfl=0.2, gpu_precision="mixed", project_path="/tmp", **extra):
    """Independent 2D Drucker-Prager slopes advanced as one problem: each slope
    gets its own region of one shared grid -- its wall at x0 (vx fixed), the
    common floor y = 0 (fixed), a far wall at x0 + L (vx fixed) with L = crest +
    run of the face + runout_factor x height -- and the regions are separated
    by gap_cells empty cells, more than the uGIMP stencil reaches, so no node
    is shared.  Every launch of the step then covers all slopes.  Each slope is
    its own material (nid = slope + 1).  Offsets are whole cells, so a slope's
    particles sit at the same place relative to the grid as when the slope is
    run alone (slope_2d_single)."""
    specs = specs if specs is not None else draw_slope_specs(n_slopes, seed, h=h, ppc=ppc)
    K, G = elastic_constants(E, nu)
    dt = cfl_dt(h, K, G, rho, cfl)
    lp = h / ppc
    x0 = 0.0
    parts, nid, slopes = [], [], []
    start = 0
    for k, sp in enumerate(specs):
        tb = math.tan(sp["beta"])
        L = sp["crest"] + sp["H"] / tb + runout_factor * sp["H"]
        L = math.ceil(L / h) * h
        pts = slope_points_2d(sp, h, ppc, jitter)
        toe0 = float(pts[:, 0].max())
        pts = pts.copy()
        pts[:, 0] += x0
        parts.append(pts)
        nid.append(np.full(len(pts), k + 1, np.int64))
        slopes.append(dict(sp, x0=x0, L=L, np=len(pts), start=start, end=start + len(pts), toe0=toe0))
        start += len(pts)
        x0 = x0 + L + gap_cells * h
    pts = np.concatenate(parts)
    nid = np.concatenate(nid)
    npart = len(pts)
    width = x0 - gap_cells * h
    top = max(s["H"] for s in slopes) + 1.0
    akw = dict(Ttol=Ttol, Te=Te, ΔT=dt, FLIP=1, PIC=0, constitutive="druckerprager", basis="uGIMP",
               device="B200", coupling="OS", scheme="MUSL", va="a", gravity=gravity, ζs=0,
               project_name="slopes2d", project_path=project_path, ϵ=precision, gpu_precision=gpu_precision,
               make_project_dir=False)
    akw.update(extra)
    args = UserArgs2D(**akw)
    grid = UserGrid2D(ϵ=precision, x1=-pad * h, x2=width + pad * h, y1=-pad * h, y2=top + pad * h,
                      dx=h, dy=h, NIC=9)
    mp = UserParticle2D(ϵ=precision, NIC=9, dx=lp, dy=lp, ξ=pts, ρs=np.full(npart, rho))
    ns = len(slopes)
    attr = UserProperty(ϵ=precision, nid=nid, ν=np.full(ns, nu), Es=np.full(ns, E), Gs=np.full(ns, G),
                        Ks=np.full(ns, K), σt=np.zeros(ns), ϕ=np.array([s["phi"] for s in slopes]),
                        ϕr=np.zeros(ns), ψ=np.full(ns, math.radians(psi_deg)),
                        c=np.array([s["c"] for s in slopes]), cr=np.zeros(ns), Hp=np.zeros(ns))
    # boundary flags: node id = ix * nny + r, r = 0 at the top (y descending)
    eps = 1e-9 * h
    vx = grid._vx
    vy = grid._vy
    wall = np.zeros(len(vx), bool)
    for s in slopes:
        wall |= np.abs(vx - s["x0"]) <= eps
        wall |= np.abs(vx - (s["x0"] + s["L"])) <= eps
    floor = vy <= eps
    fx = (wall[:, None] | floor[None, :]).ravel().astype(np.int64)
    fy = np.broadcast_to(floor[None, :], (len(vx), len(vy))).ravel().astype(np.int64)
    bc = UserVBoundary2D(ϵ=precision, vx_s_idx=fx, vx_s_val=np.zeros(grid.ni), vy_s_idx=fy,
                         vy_s_val=np.zeros(grid.ni))
    nsteps = int(math.ceil(Ttol / dt))
    return Case("slope_batch_2d", args, grid, mp, attr, bc, dt, nsteps,
                dict(np=npart, h=h, K=K, G=G, seed=seed, slopes=slopes))


def slope_2d_single(batch_case, k, **kw):
    """Slope k of a batch alone on its own grid (local frame), with the same
    particles, material and boundary layout: the plain run the batched one is
    compared with."""
    s = batch_case.meta["slopes"][k]
    a = batch_case.args
    spec = {key: s[key] for key in ("index", "target_np", "beta", "H", "crest", "c", "phi", "seed")}
    base = dict(h=batch_case.meta["h"], Ttol=a.Ttol, Te=a.Te, gpu_precision=a.gpu_precision)
    base.update(kw)
    return slope_batch_2d(specs=[spec], **base)


def slope_runouts(case, xi):
    """Per-slope run-out: the advance of the slope's farthest particle (toe)
    from its initial position, in metres."""
    out = []
    for s in case.meta["slopes"]:
        out.append(float(xi[s["start"]:s["end"], 0].max() - s["x0"] - s["toe0"]))
    return np.array(out)


def saturated_column(*, dim=2, h=0.01, ppc=2, seed=1006, jitter=0.1, size=(0.1, 0.06, 0.2), box=None, pad=2,
                     precision="FP64", constitutive="linearelastic", E=1.0e6, nu=0.3, rho_s=2650.0,
                     rho_w=1000.0, n=0.3, Kw=2.2e7, k=1.0e-3, phi_deg=30.0, c=0.0, gravity=-9.81,
                     Te=0.0, zeta_s=0.0, zeta_w=0.0, Ttol=0.05, cfl=0.2, gpu_precision="mixed",
                     project_path="/tmp", **extra):
    """Two-phase (coupling = :TS) saturated soil column of `size` (x, [y,] up)
    in a box of `box` (default: the column's own footprint, i.e. a column
    confined laterally; a wider box lets it collapse toward +x): porosity `n`,
    solid and water densities, water bulk
    modulus `Kw` and permeability `k` (the drag n·mw·g/k of P2G_TS!).  Walls
    and floor are impermeable and free-slip for both phases (normal solid and
    water velocities fixed to 0).  Δt = CFL·h / c with the undrained P-wave
    speed c = sqrt((K + 4G/3 + Kw/n) / ((1 - n) ρs))."""
    K, G = elastic_constants(E, nu)
    dt = cfl * h / math.sqrt((K + 4.0 * G / 3.0 + Kw / n) / ((1.0 - n) * rho_s))
    lp = h / ppc
    rng = np.random.Generator(np.random.PCG64(seed))
    ext = size[:2] if dim == 2 else size
    axes = [jl_range(lp / 2, lp, L - lp / 2) for L in (ext[0], ext[1]) + ((ext[2],) if dim == 3 else ())]
    bx = tuple(box) if box is not None else tuple(ext)
    pts = meshbuilder(*axes)
    pts = pts + rng.uniform(-jitter * h, jitter * h, size=pts.shape)
    npart = pts.shape[0]
    akw = dict(Ttol=Ttol, Te=Te, ΔT=dt, FLIP=1, PIC=0, constitutive=constitutive, basis="uGIMP",
               device="B200", coupling="TS", scheme="MUSL", va="a", gravity=gravity, ζs=zeta_s, ζw=zeta_w,
               project_name=f"saturated{dim}d", project_path=project_path, ϵ=precision,
               gpu_precision=gpu_precision, make_project_dir=False)
    akw.update(extra)
    mat = dict(ν=[nu], Es=[E], Gs=[G], Ks=[K], σt=[0.0], ϕ=[math.radians(phi_deg)], ϕr=[0.0], ψ=[0.0],
               c=[c], cr=[0.0], Hp=[0.0], Kw=[Kw], k=[k])
    attr = UserProperty(ϵ=precision, nid=np.ones(npart, np.int64), **mat)
    eps = 1e-9 * h
    if dim == 2:
        args = UserArgs2D(**akw)
        grid = UserGrid2D(ϵ=precision, x1=-pad * h, x2=bx[0] + pad * h, y1=-pad * h, y2=bx[1] + 3 * h,
                          dx=h, dy=h, NIC=9, phase=2)
        mp = UserParticle2D(ϵ=precision, NIC=9, dx=lp, dy=lp, ξ=pts, ρs=np.full(npart, rho_s), phase=2,
                            n=np.full(npart, n), ρw=np.full(npart, rho_w))
        gx, gy = grid.xi[:, 0], grid.xi[:, 1]
        fx = ((gx <= eps) | (gx >= bx[0] - eps)).astype(np.int64)
        fy = (gy <= eps).astype(np.int64)
        z = np.zeros(grid.ni)
        bc = UserVBoundary2D(ϵ=precision, vx_s_idx=fx, vx_s_val=z, vy_s_idx=fy, vy_s_val=z,
                             vx_w_idx=fx, vx_w_val=z, vy_w_idx=fy, vy_w_val=z)
    else:
        args = UserArgs3D(**akw)
        grid = UserGrid3D(ϵ=precision, x1=-pad * h, x2=bx[0] + pad * h, y1=-pad * h, y2=bx[1] + pad * h,
                          z1=-pad * h, z2=bx[2] + 3 * h, dx=h, dy=h, dz=h, NIC=27, phase=2)
        mp = UserParticle3D(ϵ=precision, NIC=27, dx=lp, dy=lp, dz=lp, ξ=pts, ρs=np.full(npart, rho_s),
                            phase=2, n=np.full(npart, n), ρw=np.full(npart, rho_w))
        gx, gy, gz = grid.xi[:, 0], grid.xi[:, 1], grid.xi[:, 2]
        fx = ((gx <= eps) | (gx >= bx[0] - eps)).astype(np.int64)
        fy = ((gy <= eps) | (gy >= bx[1] - eps)).astype(np.int64)
        fz = (gz <= eps).astype(np.int64)
        z = np.zeros(grid.ni)
        bc = UserVBoundary3D(ϵ=precision, vx_s_idx=fx, vx_s_val=z, vy_s_idx=fy, vy_s_val=z, vz_s_idx=fz,
                             vz_s_val=z, vx_w_idx=fx, vx_w_val=z, vy_w_idx=fy, vy_w_val=z, vz_w_idx=fz,
                             vz_w_val=z)
    nsteps = int(math.ceil(Ttol / dt))
    return Case(f"saturated_column_{dim}d", args, grid, mp, attr, bc, dt, nsteps,
                dict(np=npart, h=h, K=K, G=G, seed=seed, height=ext[-1], rho_w=rho_w, n=n))


def collapse_2d_validation(*, precision="FP64", gpu_precision="mixed", Ttol=1.0, project_path="/tmp", **extra):
    """The reference's 2D granular column validation case (test/validation/2d_case.jl):
    a 0.2 x 0.1 m column of sand (K = 7e5 Pa, ν = 0.3, ρ = 2650, Drucker-Prager
    φ = 19.8°, c = 0) on a 2.5 mm grid over [-0.025, 0.82] x [-0.025, 0.12],
    2 x 2 particles per cell on a regular lattice (12 800 particles), walls at
    x <= 0 and x >= 0.8 and a rough floor (both velocity components fixed at
    y <= 0), gravity -9.8, Δt = 0.5 h / sqrt(E/ρ), 1 s.  Its final free surface
    is compared with laboratory measurements shipped with the reference."""
    h = 0.0025
    K, nu, rho = 7e5, 0.3, 2650.0
    E = K * (3.0 * (1.0 - 2.0 * nu))
    G = E / (2.0 * (1.0 + nu))
    dt = 0.5 * h / math.sqrt(E / rho)
    lp = h / 2
    pts = meshbuilder(jl_range(lp / 2, lp, 0.2 - lp / 2), jl_range(lp / 2, lp, 0.1 - lp / 2))
    npart = pts.shape[0]
    akw = dict(Ttol=Ttol, Te=0, ΔT=dt, FLIP=1, PIC=0, constitutive="druckerprager", basis="uGIMP",
               device="B200", coupling="OS", scheme="MUSL", va="a", gravity=-9.8, ζs=0,
               project_name="collapse2d_validation", project_path=project_path, ϵ=precision,
               gpu_precision=gpu_precision, make_project_dir=False)
    akw.update(extra)
    args = UserArgs2D(**akw)
    grid = UserGrid2D(ϵ=precision, x1=-0.025, x2=0.82, y1=-0.025, y2=0.12, dx=h, dy=h, NIC=9)
    mp = UserParticle2D(ϵ=precision, NIC=9, dx=lp, dy=lp, ξ=pts, ρs=np.full(npart, rho))
    attr = UserProperty(ϵ=precision, nid=np.ones(npart, np.int64), ν=[nu], Es=[E], Gs=[G], Ks=[K],
                        σt=[0.0], ϕ=[math.radians(19.8)], ϕr=[0.0], ψ=[0.0], c=[0.0], cr=[0.0], Hp=[0.0])
    gx, gy = grid.xi[:, 0], grid.xi[:, 1]
    vx = ((gx <= 0.0) | (gx >= 0.8) | (gy <= 0.0)).astype(np.int64)
    vy = (gy <= 0.0).astype(np.int64)
    bc = UserVBoundary2D(ϵ=precision, vx_s_idx=vx, vx_s_val=np.zeros(grid.ni), vy_s_idx=vy,
                         vy_s_val=np.zeros(grid.ni))
    nsteps = int(math.ceil(Ttol / dt))
    return Case("collapse_2d_validation", args, grid, mp, attr, bc, dt, nsteps, dict(np=npart, h=h, K=K, G=G, seed=0))


def collapse_3d_validation(*, precision="FP64", gpu_precision="mixed", Ttol=1.0, project_path="/tmp", **extra):
    """The reference's 3D granular column validation case (test/validation/3d_case.jl):
    the 2D case as a 0.05 m thick slab -- a 0.05 x 0.2 x 0.1 m column (x across,
    y along the flume, z up) of sand (K = 7e5 Pa, ν = 0.3, ρ = 2650,
    Drucker-Prager φ = 19.8°, c = 0) on a 2.5 mm grid over [-0.02, 0.07] x
    [-0.02, 0.75] x [-0.02, 0.12], 2 x 2 x 2 particles per cell (512 000
    particles), USL scheme, free-slip side walls at x <= 0 and x >= 0.05, a wall
    at y <= 0 (x and y fixed), a rough floor at z <= 0 (all fixed), gravity
    -9.8, Δt = 0.5 h / sqrt(E/ρ), 1 s."""
    h = 0.0025
    K, nu, rho = 7e5, 0.3, 2650.0
    E = K * (3.0 * (1.0 - 2.0 * nu))
    G = E / (2.0 * (1.0 + nu))
    dt = 0.5 * h / math.sqrt(E / rho)
    lp = h / 2
    pts = meshbuilder(jl_range(lp / 2, lp, 0.05 - lp / 2), jl_range(lp / 2, lp, 0.2 - lp / 2),
                      jl_range(lp / 2, lp, 0.1 - lp / 2))
    npart = pts.shape[0]
    akw = dict(Ttol=Ttol, Te=0, ΔT=dt, FLIP=1, PIC=0, constitutive="druckerprager", basis="uGIMP",
               device="B200", coupling="OS", scheme="USL", va="a", gravity=-9.8, ζs=0,
               project_name="collapse3d_validation", project_path=project_path, ϵ=precision,
               gpu_precision=gpu_precision, make_project_dir=False)
    akw.update(extra)
    args = UserArgs3D(**akw)
    grid = UserGrid3D(ϵ=precision, x1=-0.02, x2=0.07, y1=-0.02, y2=0.75, z1=-0.02, z2=0.12, dx=h, dy=h, dz=h,
                      NIC=27)
    mp = UserParticle3D(ϵ=precision, NIC=27, dx=lp, dy=lp, dz=lp, ξ=pts, ρs=np.full(npart, rho))
    attr = UserProperty(ϵ=precision, nid=np.ones(npart, np.int64), ν=[nu], Es=[E], Gs=[G], Ks=[K],
                        σt=[0.0], ϕ=[math.radians(19.8)], ϕr=[0.0], ψ=[0.0], c=[0.0], cr=[0.0], Hp=[0.0])
    gx, gy, gz = grid.xi[:, 0], grid.xi[:, 1], grid.xi[:, 2]
    vx = ((gx <= 0.0) | (gx >= 0.05) | (gz <= 0.0) | (gy <= 0.0)).astype(np.int64)
    vy = ((gy <= 0.0) | (gz <= 0.0)).astype(np.int64)
    vz = (gz <= 0.0).astype(np.int64)
    z = np.zeros(grid.ni)
    bc = UserVBoundary3D(ϵ=precision, vx_s_idx=vx, vx_s_val=z, vy_s_idx=vy, vy_s_val=z.copy(), vz_s_idx=vz,
                         vz_s_val=z.copy())
    nsteps = int(math.ceil(Ttol / dt))
    return Case("collapse_3d_validation", args, grid, mp, attr, bc, dt, nsteps, dict(np=npart, h=h, K=K, G=G, seed=0))


def collapse_2d_example(*, precision="FP64", gpu_precision="mixed", Ttol=1.0, project_path="/tmp", **extra):
    """The reference's 2D column-collapse example (examples/2d_collapse.ipynb),
    the case behind its published 2D throughput (2.11e3 it/s, FP64, on an
    unstated NVIDIA GPU): a 0.2 x 0.1 m column, 2 x 2 particles per 2 mm cell
    (20 000 particles) on [-0.1, 0.82] x [-0.1, 0.12] (51 171 nodes),
    Drucker-Prager φ = 19.8°, c = 0, ψ = 0, K = 7e5 Pa, ν = 0.3, ρ = 2650,
    MUSL va = :a, gravity -9.8, Δt = 0.5 h / sqrt(E/ρ), 1 s; walls at x <= 0 and
    x >= 0.8 and a rough floor (both components fixed at y <= 0)."""
    h = 0.002
    K, nu, rho = 7e5, 0.3, 2650.0
    E = K * (3.0 * (1.0 - 2.0 * nu))
    G = E / (2.0 * (1.0 + nu))
    dt = 0.5 * h / math.sqrt(E / rho)
    lp = h / 2
    pts = meshbuilder(jl_range(lp / 2, lp, 0.2 - lp / 2), jl_range(lp / 2, lp, 0.1 - lp / 2))
    npart = pts.shape[0]
    akw = dict(Ttol=Ttol, Te=0, ΔT=dt, FLIP=1, PIC=0, constitutive="druckerprager", basis="uGIMP",
               device="B200", coupling="OS", scheme="MUSL", va="a", gravity=-9.8, ζs=0,
               project_name="2d_collapse", project_path=project_path, ϵ=precision,
               gpu_precision=gpu_precision, make_project_dir=False)
    akw.update(extra)
    args = UserArgs2D(**akw)
    grid = UserGrid2D(ϵ=precision, x1=-0.1, x2=0.82, y1=-0.1, y2=0.12, dx=h, dy=h, NIC=9)
    mp = UserParticle2D(ϵ=precision, NIC=9, dx=lp, dy=lp, ξ=pts, ρs=np.full(npart, rho))
    attr = UserProperty(ϵ=precision, nid=np.ones(npart, np.int64), ν=[nu], Es=[E], Gs=[G], Ks=[K],
                        σt=[0.0], ϕ=[math.radians(19.8)], ϕr=[0.0], ψ=[0.0], c=[0.0], cr=[0.0], Hp=[0.0])
    gx, gy = grid.xi[:, 0], grid.xi[:, 1]
    vx = ((gx <= 0.0) | (gx >= 0.8) | (gy <= 0.0)).astype(np.int64)
    vy = (gy <= 0.0).astype(np.int64)
    bc = UserVBoundary2D(ϵ=precision, vx_s_idx=vx, vx_s_val=np.zeros(grid.ni), vy_s_idx=vy,
                         vy_s_val=np.zeros(grid.ni))
    nsteps = int(math.ceil(Ttol / dt))
    return Case("collapse_2d_example", args, grid, mp, attr, bc, dt, nsteps, dict(np=npart, h=h, K=K, G=G, seed=0))


def collapse_3d_example(*, precision="FP64", gpu_precision="mixed", Ttol=1.0, mvl=True, project_path="/tmp",
                        **extra):
    """The reference's 3D column-collapse example (examples/3d_collapse.ipynb),
    the case behind its published 3D throughput (66.3 it/s, FP64, on an
    unstated NVIDIA GPU): a 0.05 x 0.2 x 0.1 m column, 2 x 2 x 2 particles per
    2.5 mm cell (512 000 particles) on [-0.02, 0.07] x [-0.02, 0.55] x
    [-0.02, 0.12] (482 961 nodes), Drucker-Prager φ = 19.8°, c = 0, ψ = 0,
    E = 1 MPa, ν = 0, ρ = 2700, MUSL va = :a, MVL on, gravity -9.8,
    Δt = 0.5 h / sqrt((K + 4G/3)/ρ), 1 s; free-slip side walls at x <= 0 and
    x >= 0.05, a wall at y <= 0 (x and y fixed), a rough floor."""
    h = 0.0025
    E, nu, rho = 1.0e6, 0.0, 2700.0
    K, G = elastic_constants(E, nu)
    dt = 0.5 * h / math.sqrt((K + 4.0 / 3.0 * G) / rho)
    lp = h / 2
    pts = meshbuilder(jl_range(lp / 2, lp, 0.05 - lp / 2), jl_range(lp / 2, lp, 0.2 - lp / 2),
                      jl_range(lp / 2, lp, 0.1 - lp / 2))
    npart = pts.shape[0]
    akw = dict(Ttol=Ttol, Te=0, ΔT=dt, FLIP=1, PIC=0, constitutive="druckerprager", basis="uGIMP",
               device="B200", coupling="OS", scheme="MUSL", va="a", gravity=-9.8, ζs=0, MVL=mvl,
               project_name="3d_collapse", project_path=project_path, ϵ=precision,
               gpu_precision=gpu_precision, make_project_dir=False)
    akw.update(extra)
    args = UserArgs3D(**akw)
    grid = UserGrid3D(ϵ=precision, x1=-0.02, x2=0.07, y1=-0.02, y2=0.55, z1=-0.02, z2=0.12, dx=h, dy=h, dz=h,
                      NIC=27)
    mp = UserParticle3D(ϵ=precision, NIC=27, dx=lp, dy=lp, dz=lp, ξ=pts, ρs=np.full(npart, rho))
    attr = UserProperty(ϵ=precision, nid=np.ones(npart, np.int64), ν=[nu], Es=[E], Gs=[G], Ks=[K],
                        σt=[0.0], ϕ=[math.radians(19.8)], ϕr=[0.0], ψ=[0.0], c=[0.0], cr=[0.0], Hp=[0.0])
    gx, gy, gz = grid.xi[:, 0], grid.xi[:, 1], grid.xi[:, 2]
    vx = ((gx <= 0.0) | (gx >= 0.05) | (gz <= 0.0) | (gy <= 0.0)).astype(np.int64)
    vy = ((gy <= 0.0) | (gz <= 0.0)).astype(np.int64)
    vz = (gz <= 0.0).astype(np.int64)
    z = np.zeros(grid.ni)
    bc = UserVBoundary3D(ϵ=precision, vx_s_idx=vx, vx_s_val=z, vy_s_idx=vy, vy_s_val=z.copy(), vz_s_idx=vz,
                         vz_s_val=z.copy())
    nsteps = int(math.ceil(Ttol / dt))
    return Case("collapse_3d_example", args, grid, mp, attr, bc, dt, nsteps, dict(np=npart, h=h, K=K, G=G, seed=0))


def cantilever_2d(*, precision="FP64", gpu_precision="fp64", Ttol=3.0, dt=1e-4, constitutive="linearelastic",
                  project_path="/tmp", **extra):
    """The reference's 2D cantilever beam (test/c1_accuracy/t1_cantilever_beam/
    2d_cantilever_beam.jl): a 4 x 1 m beam (E = 1 MPa, ν = 0.3, ρ = 1050) on a
    0.25 m grid over [-3, 8] x [-8, 4], 3 x 3 particles per cell, clamped where
    nodes have x <= 0 and y >= -1 (both velocity components fixed), gravity
    -9.8, Δt = 1e-4, 3 s, MUSL, FLIP 1.  The reference runs it with its
    Neo-Hookean model and plots the deflection of the bottom corner particle at
    the free end against FEM and MPM curves it ships; this backend provides the
    linear elastic model (with the Jaumann rotation of liE!).  meta["tip"] is
    that particle's index."""
    h, E, nu, rho = 0.25, 1.0e6, 0.3, 1050.0
    K, G = elastic_constants(E, nu)
    lp = h / 3
    pts = meshbuilder(jl_range(lp / 2, lp, 4.0 - lp / 2), jl_range(lp / 2, lp, 1.0 - lp / 2))
    npart = pts.shape[0]
    akw = dict(Ttol=Ttol, Te=0, ΔT=dt, FLIP=1, PIC=0, constitutive=constitutive, basis="uGIMP",
               device="B200", coupling="OS", scheme="MUSL", va="a", gravity=-9.8, ζs=0,
               project_name="2d_cantilever_beam", project_path=project_path, ϵ=precision,
               gpu_precision=gpu_precision, make_project_dir=False)
    akw.update(extra)
    args = UserArgs2D(**akw)
    grid = UserGrid2D(ϵ=precision, x1=-3.0, x2=8.0, y1=-8.0, y2=4.0, dx=h, dy=h, NIC=9)
    mp = UserParticle2D(ϵ=precision, NIC=9, dx=lp, dy=lp, ξ=pts, ρs=np.full(npart, rho))
    attr = UserProperty(ϵ=precision, nid=np.ones(npart, np.int64), ν=[nu], Es=[E], Gs=[G], Ks=[K],
                        σt=[0.0], ϕ=[0.0], ϕr=[0.0], ψ=[0.0], c=[0.0], cr=[0.0], Hp=[0.0])
    gx, gy = grid.xi[:, 0], grid.xi[:, 1]
    clamp = ((gx <= 0.0) & (gy >= -1.0)).astype(np.int64)
    bc = UserVBoundary2D(ϵ=precision, vx_s_idx=clamp, vx_s_val=np.zeros(grid.ni), vy_s_idx=clamp.copy(),
                         vy_s_val=np.zeros(grid.ni))
    low = pts[:, 1] == pts[:, 1].min()
    tip = int(np.nonzero(low & (pts[:, 0] == pts[low, 0].max()))[0][0])
    nsteps = int(round(Ttol / dt))
    return Case("cantilever_2d", args, grid, mp, attr, bc, dt, nsteps, dict(np=npart, h=h, K=K, G=G, tip=tip))


def free_surface(xi, x_edges):
    """Height of the deposit per x bin: the highest particle in each bin
    (NaN for empty bins)."""
    x, y = xi[:, 0], xi[:, 1]
    k = np.digitize(x, x_edges) - 1
    out = np.full(len(x_edges) - 1, np.nan)
    for b in range(len(x_edges) - 1):
        sel = k == b
        if sel.any():
            out[b] = y[sel].max()
    return out
