"""Host-side mirrors of MaterialPointSolver.jl's user structs.

Each constructor follows the reference's keyword constructor of the same name
(argument names, defaults, validation and array shapes), so a script written
against the reference reads the same here.  Arrays are numpy arrays in the
reference's memory layout: Julia column-major ``n x k`` matrices become
Fortran-ordered ``(n, k)`` arrays, i.e. one contiguous column per component
(structure-of-arrays), which is what the C-ABI library consumes directly.

Julia field names that are not ASCII identifiers are transliterated:

=========  ==========  =========  ==========
reference  here        reference  here
=========  ==========  =========  ==========
ξ          xi          ϵijs       eps
ξ0         xi0         Δϵijs      deps
σij        sig         ϵq         epsq
σm         sigm        ϵk         epsk
Ω          Omega       ϵv         epsv
Ω0         Omega0      ΔFs        dF
ρs         rho         ∂Nx/y/z    dNx/dNy/dNz
ρs0        rho0        ΔT         dT
ζs         zeta_s      ϵ (prec.)  precision
ϕ          phi         ψ          psi
σt         sigt        ν          nu
=========  ==========  =========  ==========

Keyword arguments may also be given under their Julia spelling (``ΔT=…``,
``ζs=…``, ``ϵ="FP32"``, ``ξ=…``, ``ρs=…``, ``ϕ=…``); they are mapped to the
names above.
"""
from __future__ import annotations

import os
import shutil
import unicodedata

import numpy as np

_ALIASES = {
    "ΔT": "dT", "ζs": "zeta_s", "ζw": "zeta_w", "αT": "alphaT", "ϵ": "precision",
    "ξ": "xi", "ρs": "rho", "ρw": "rho_w", "ν": "nu", "ϕ": "phi", "ϕr": "phi_r",
    "ψ": "psi", "σt": "sigt",
}
_ALIASES = {unicodedata.normalize("NFKC", k): v for k, v in _ALIASES.items()}


def _norm_kwargs(kw):
    out = {}
    for k, v in kw.items():
        k2 = _ALIASES.get(unicodedata.normalize("NFKC", k), k)
        out[k2] = v
    return out


def _types(precision):
    """T1/T2 selection of the reference (modelargs.jl:65-66, grid.jl:88-90)."""
    if precision == "FP32":
        return np.int32, np.float32
    return np.int64, np.float64


def _f(a, dtype):
    return np.asfortranarray(np.asarray(a, dtype=dtype))


# ---------------------------------------------------------------------------
# Args2D / Args3D  (src/types/modelargs.jl:31-98, 122-189)
# ---------------------------------------------------------------------------
class Args:
    dim = 0

    def __init__(self, **kw):
        kw = _norm_kwargs(kw)
        required = ("Ttol", "dT", "constitutive", "project_name", "project_path")
        for r in required:
            if r not in kw:
                raise TypeError(f"missing keyword argument {r}")
        self.Ttol = float(kw["Ttol"])
        self.Te = float(kw.get("Te", 0))
        self.dT = float(kw["dT"])
        self.time_step = kw.get("time_step", "fixed")
        self.FLIP = float(kw.get("FLIP", 1))
        self.PIC = float(kw.get("PIC", 0))
        self.constitutive = kw["constitutive"]
        self.basis = kw.get("basis", "uGIMP")
        self.animation = bool(kw.get("animation", False))
        self.hdf5 = bool(kw.get("hdf5", False))
        self.hdf5_step = int(kw.get("hdf5_step", 1))
        self.MVL = bool(kw.get("MVL", False))
        self.device = kw.get("device", "CPU")
        self.coupling = kw.get("coupling", "OS")
        self.scheme = kw.get("scheme", "MUSL")
        self.va = kw.get("va", "a")
        self.progressbar = bool(kw.get("progressbar", True))
        self.gravity = float(kw.get("gravity", -9.8))
        self.zeta_s = float(kw.get("zeta_s", 0))
        self.zeta_w = float(kw.get("zeta_w", 0))
        self.alphaT = float(kw.get("alphaT", 0.5))
        self.iter_num = int(kw.get("iter_num", 0))
        self.end_time = float(kw.get("end_time", 0))
        self.start_time = float(kw.get("start_time", 0))
        self.project_name = kw["project_name"]
        self.project_path = kw["project_path"]
        self.precision = kw.get("precision", "FP64")
        # B200 backend options (no reference counterpart): arithmetic of the
        # device step ("mixed" = FP32 bulk with FP64 positions / determinant,
        # "fp64" = all FP64 for self-checks), the 3D Mohr-Coulomb mode and the
        # particle re-sort period.
        self.gpu_precision = kw.get("gpu_precision", "mixed")
        self.mc3d = kw.get("mc3d", "literal")
        self.sort_every = int(kw.get("sort_every", 0))
        self.T1, self.T2 = _types(self.precision)
        # parameter checks, modelargs.jl:76-91
        cop_set = ["OS", "TS"]
        bas_set = ["uGIMP", "linear", "gslinear"]
        dev_set = ["CPU", "CUDA", "ROCm", "oneAPI", "Metal", "B200"]
        if not 0 < self.Ttol:
            raise ValueError("Simulation time cannot be ≤0 s.")
        if not self.dT <= self.Ttol:
            raise ValueError(f"Time step cannot be >{self.Ttol}s.")
        if not 0 <= self.Te <= self.Ttol:
            raise ValueError(f"Elastic loading time must in 0~{self.Ttol}s.")
        if self.basis not in bas_set:
            raise ValueError(f"Cannot find {self.basis} basis function.")
        if (self.FLIP + self.PIC) != 1:
            raise ValueError("FLIP+PIC must be 1.")
        if not 0 <= self.alphaT <= 1:
            raise ValueError("Time step factor error.")
        if not 0 <= self.zeta_s <= 1:
            raise ValueError("Out of range 0≤ζs≤1.")
        if not 0 <= self.zeta_w <= 1:
            raise ValueError("Out of range 0≤ζw≤1.")
        if self.project_name == "":
            raise ValueError("Empty project name.")
        if self.coupling not in cop_set:
            raise ValueError("Coupling mode is wrong.")
        if self.device not in dev_set:
            raise ValueError(f"Cannot find {self.device} device.")
        if self.time_step not in ("fixed", "auto"):
            raise ValueError(f"{self.time_step} time step is not allowed.")
        if self.va not in ("v", "a"):
            raise ValueError(f"Cannot find {self.va} velocity update mode.")
        if self.animation and not self.hdf5:
            self.hdf5 = True
        if self.hdf5 and self.hdf5_step <= 0:
            raise ValueError("HDF5 step cannot be ≤0.")
        folder = os.path.join(os.path.abspath(self.project_path), self.project_name)
        if kw.get("make_project_dir", True):
            os.makedirs(folder, exist_ok=True)
            shutil.rmtree(folder, ignore_errors=True)
            os.makedirs(folder, exist_ok=True)


class Args2D(Args):
    dim = 2


class Args3D(Args):
    dim = 3


def UserArgs2D(**kw):
    return Args2D(**kw)


def UserArgs3D(**kw):
    return Args3D(**kw)


# ---------------------------------------------------------------------------
# Grid2D / Grid3D  (src/types/grid.jl:33-145, 170-309)
# ---------------------------------------------------------------------------
def _axis(a1, a2, h):
    """Nodes of the Julia range a1:h:a2 (values a1 + i*h; the last node is the
    largest one not beyond a2, allowing for round-off like Julia's range)."""
    n = int(np.floor((a2 - a1) / h * (1 + 1e-12) + 1e-9)) + 1
    return a1 + np.arange(n, dtype=np.float64) * h


class Grid:
    dim = 0


class Grid2D(Grid):
    """Node order as the reference: x-major columns, y DESCENDING inside a
    column (grid.jl:92-100): node id (1-based) = ix*nny + r + 1, r = 0 at y2."""
    dim = 2

    def __init__(self, *, precision="FP64", phase=1, x1, x2, y1, y2, dx, dy, NIC=9, ext=0):
        if not x1 < x2:
            raise ValueError("x1 should be less than x2")
        if not y1 < y2:
            raise ValueError("y1 should be less than y2")
        if not (dx > 0 and dy > 0):
            raise ValueError("dx and dy should be positive")
        self.T1, self.T2 = _types(precision)
        self.precision = precision
        self.phase = phase if phase in (1, 2) else 1
        self.NIC = NIC if NIC in (4, 9) else 9
        self.x1, self.x2, self.y1, self.y2 = float(x1), float(x2), float(y1), float(y2)
        self.dx, self.dy = float(dx), float(dy)
        vx = _axis(self.x1, self.x2, self.dx)
        vy = _axis(self.y1, self.y2, self.dy)[::-1]
        self.nnx, self.nny = len(vx), len(vy)
        self.ni = self.nnx * self.nny
        self._vx, self._vy = vx, vy   # vy descending, as stored
        self._xi = None
        self.ncx, self.ncy = self.nnx - 1, self.nny - 1
        self.nc = self.ncx * self.ncy
        T2 = self.T2
        self.sigm = np.zeros(self.nc, T2)
        self.Omega = np.zeros(self.nc, T2)

    @property
    def xi(self):
        # node coordinates (ni x 2), built on first use
        if self._xi is None:
            x = np.repeat(self._vx, self.nny)
            y = np.tile(self._vy, self.nnx)
            self._xi = _f(np.stack([x, y], axis=1), self.T2)
        return self._xi

    def __getattr__(self, name):
        # the reference's grid work arrays, allocated on first use
        if name in ("ms",):
            arr = np.zeros(self.ni, self.T2)
        elif name in ("ps", "vs", "vsT", "as_", "fs", "dus"):
            arr = _f(np.zeros((self.ni, 2)), self.T2)
        else:
            raise AttributeError(name)
        object.__setattr__(self, name, arr)
        return arr


class Grid3D(Grid):
    """Node order as the reference: y fastest, then x, then z (grid.jl:236-249)."""
    dim = 3

    def __init__(self, *, precision="FP64", phase=1, x1, x2, y1, y2, z1, z2, dx, dy, dz,
                 NIC=27, ext=0):
        if not x1 < x2:
            raise ValueError("x1 should be less than x2")
        if not y1 < y2:
            raise ValueError("y1 should be less than y2")
        if not z1 < z2:
            raise ValueError("z1 should be less than z2")
        if not (dx > 0 and dy > 0 and dz > 0):
            raise ValueError("dx, dy, and dz should be positive")
        self.T1, self.T2 = _types(precision)
        self.precision = precision
        self.phase = phase if phase in (1, 2) else 1
        self.NIC = NIC if NIC in (8, 27) else 27
        self.x1, self.x2, self.y1, self.y2 = float(x1), float(x2), float(y1), float(y2)
        self.z1, self.z2 = float(z1), float(z2)
        self.dx, self.dy, self.dz = float(dx), float(dy), float(dz)
        vx = _axis(self.x1, self.x2, self.dx)
        vy = _axis(self.y1, self.y2, self.dy)
        vz = _axis(self.z1, self.z2, self.dz)
        self.nnx, self.nny, self.nnz = len(vx), len(vy), len(vz)
        self.ni = self.nnx * self.nny * self.nnz
        self.ncx, self.ncy, self.ncz = self.nnx - 1, self.nny - 1, self.nnz - 1
        self.nc = self.ncx * self.ncy * self.ncz
        self._vx, self._vy, self._vz = vx, vy, vz
        self._xi = None
        T2 = self.T2
        self.sigm = np.zeros(self.nc, T2)
        self.Omega = np.zeros(self.nc, T2)
        self._node_arrays = ("ms", "ps", "vs", "vsT", "as_", "fs", "dus")

    @property
    def xi(self):
        # node coordinates (ni x 3), built on first use: large grids never
        # need them on the host when the device computes node positions.
        if self._xi is None:
            Z, X, Y = np.meshgrid(self._vz, self._vx, self._vy, indexing="ij")
            self._xi = _f(np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1), self.T2)
        return self._xi

    def __getattr__(self, name):
        # grid work arrays of the reference (ms, ps, vs, vsT, as, fs, Δus) are
        # allocated lazily: the B200 backend keeps its own device grid.
        if name in ("ms",):
            arr = np.zeros(self.ni, self.T2)
        elif name in ("ps", "vs", "vsT", "as_", "fs", "dus"):
            arr = _f(np.zeros((self.ni, 3)), self.T2)
        else:
            raise AttributeError(name)
        object.__setattr__(self, name, arr)
        return arr


def UserGrid2D(*, ϵ="FP64", **kw):
    kw = _norm_kwargs(kw)
    return Grid2D(precision=kw.pop("precision", ϵ), **kw)


def UserGrid3D(*, ϵ="FP64", **kw):
    kw = _norm_kwargs(kw)
    return Grid3D(precision=kw.pop("precision", ϵ), **kw)


# ---------------------------------------------------------------------------
# Particle2D / Particle3D  (src/types/particle.jl:33-138, 160-271)
# ---------------------------------------------------------------------------
class Particle:
    dim = 0

    def _init(self, D, precision, NIC, lps, xi, rho, phase):
        T1, T2 = _types(precision)
        self.T1, self.T2 = T1, T2
        self.precision = precision
        self.phase = phase if phase in (1, 2) else 1
        xi = np.asarray(xi, dtype=np.float64)
        if xi.ndim != 2 or xi.shape[1] != D:
            raise ValueError(f"ξ should have {D} columns")
        npart = xi.shape[0]
        self.np = npart
        self.NIC = NIC
        vol = float(np.prod(lps))
        self.Omega0 = np.full(npart, vol, T2)
        self.Omega = self.Omega0.copy()
        nv = 4 if D == 2 else 6
        eye = np.eye(D).ravel()
        self.F = _f(np.tile(eye, (npart, 1)), T2)
        self.xi = np.array(xi, dtype=T2, order="F")   # own copy, like the reference's struct
        self.xi0 = self.xi.copy(order="F")
        self.rho = np.asarray(rho, T2).copy()
        if self.rho.shape != (npart,):
            raise ValueError("ρs must have one entry per particle")
        self.rho0 = self.rho.copy()
        self.p2c = np.zeros(npart, T1)
        self.ms = np.zeros(npart, T2)
        self.epsq = np.zeros(npart, T2)
        self.epsk = np.zeros(npart, T2)
        self.epsv = np.zeros(npart, T2)
        self.sigm = np.zeros(npart, T2)
        for name in ("eps", "sig", "deps", "sij"):
            setattr(self, name, _f(np.zeros((npart, nv)), T2))
        self.dF = _f(np.zeros((npart, D * D)), T2)
        self.ps = _f(np.zeros((npart, D)), T2)
        self.vs = _f(np.zeros((npart, D)), T2)

    def _init_water(self, n, rho_w):
        """Two-phase fields (particle.jl:103-128): per particle when phase = 2,
        single-entry placeholders otherwise."""
        D, T1, T2, npart = self.dim, self.T1, self.T2, self.np
        nv = 4 if D == 2 else 6
        n = np.zeros(1) if n is None else np.asarray(n, np.float64).ravel()
        rho_w = np.zeros(1) if rho_w is None else np.asarray(rho_w, np.float64).ravel()
        k, dof = (npart, D) if self.phase == 2 else (1, 1)
        if self.phase == 2:
            if n.shape == (1,):
                n = np.full(npart, n[0])
            if rho_w.shape == (1,):
                rho_w = np.full(npart, rho_w[0])
            if n.shape != (npart,) or rho_w.shape != (npart,):
                raise ValueError("n and ρw must have one entry per particle")
        self.n = np.asarray(n, T2).copy()
        self.rho_w = np.asarray(rho_w, T2).copy()
        self.rho_w0 = self.rho_w.copy()
        self.mw = np.zeros(k, T2)
        self.mi = np.zeros(k, T2)
        self.sigw = np.zeros(k, T2)
        self.epsw = _f(np.zeros((k, nv)), T2)
        self.depsw = _f(np.zeros((k, nv)), T2)
        self.vw = _f(np.zeros((k, dof)), T2)
        self.pw = _f(np.zeros((k, dof)), T2)

    def alloc_weights(self):
        """The reference's per-particle stencil tables (p2n, Nij, ∂N*); only the
        oracle fills them, the device recomputes weights instead of storing them."""
        npart, NIC = self.np, self.NIC
        self.p2n = _f(np.zeros((npart, NIC)), self.T1)
        self.Nij = _f(np.zeros((npart, NIC)), self.T2)
        self.dNx = _f(np.zeros((npart, NIC)), self.T2)
        self.dNy = _f(np.zeros((npart, NIC)), self.T2)
        if self.dim == 3:
            self.dNz = _f(np.zeros((npart, NIC)), self.T2)


class Particle2D(Particle):
    dim = 2

    def __init__(self, *, precision="FP64", phase=1, NIC=9, dx, dy, xi, rho, n=None, rho_w=None, ext=0):
        if not (dx > 0 and dy > 0):
            raise ValueError("dx and dy should be positive")
        self.dx, self.dy = float(dx), float(dy)
        self._init(2, precision, NIC if NIC in (4, 9) else 9, (dx, dy), xi, rho, phase)
        self._init_water(n, rho_w)


class Particle3D(Particle):
    dim = 3

    def __init__(self, *, precision="FP64", phase=1, NIC=27, dx, dy, dz, xi, rho, n=None, rho_w=None,
                 ext=0):
        if not (dx > 0 and dy > 0 and dz > 0):
            raise ValueError("dx, dy, and dz should be positive")
        self.dx, self.dy, self.dz = float(dx), float(dy), float(dz)
        self._init(3, precision, NIC if NIC in (8, 27) else 27, (dx, dy, dz), xi, rho, phase)
        self._init_water(n, rho_w)


def UserParticle2D(*, ϵ="FP64", **kw):
    kw = _norm_kwargs(kw)
    return Particle2D(precision=kw.pop("precision", ϵ), **kw)


def UserParticle3D(*, ϵ="FP64", **kw):
    kw = _norm_kwargs(kw)
    return Particle3D(precision=kw.pop("precision", ϵ), **kw)


# ---------------------------------------------------------------------------
# Property  (src/types/property.jl:31-72)
# ---------------------------------------------------------------------------
class Property:
    def __init__(self, *, precision="FP64", nid, nu, Es, Gs, Ks, Kw=(0,), k=(0,), sigt=(0,),
                 phi=(0,), phi_r=(0,), psi=(0,), c=(0,), cr=(0,), Hp=(0,), ext=0):
        T1, T2 = _types(precision)
        if not (len(Es) == len(Gs) == len(Ks) == len(nu)):
            raise ValueError("The length of Es, Gs, Ks, and ν must be the same.")
        nid = np.asarray(nid)
        if len(np.unique(nid)) != len(Es):
            raise ValueError("nid layer must be the same as the length of properties.")
        self.T1, self.T2 = T1, T2
        self.nid = nid.astype(T1)
        self.nu = np.asarray(nu, T2)
        self.Es = np.asarray(Es, T2)
        self.Gs = np.asarray(Gs, T2)
        self.Ks = np.asarray(Ks, T2)
        nmat = len(Es)

        def per_mat(a):
            a = np.asarray(a, T2)
            if a.shape == (1,) and nmat > 1:
                a = np.full(nmat, a[0], T2)
            return a

        self.sigt = per_mat(sigt)
        self.phi = per_mat(phi)
        self.phi_r = per_mat(phi_r)
        self.psi = per_mat(psi)
        self.c = per_mat(c)
        self.cr = per_mat(cr)
        self.Hp = per_mat(Hp)
        self.Kw = np.asarray(Kw, T2)
        self.k = np.asarray(k, T2)


def UserProperty(*, ϵ="FP64", **kw):
    kw = _norm_kwargs(kw)
    return Property(precision=kw.pop("precision", ϵ), **kw)


# ---------------------------------------------------------------------------
# VBoundary2D / VBoundary3D  (src/types/boundary.jl:33-131)
# ---------------------------------------------------------------------------
class VBoundary:
    pass


class VBoundary2D(VBoundary):
    dim = 2

    def __init__(self, *, precision="FP64", vx_s_idx, vx_s_val, vy_s_idx, vy_s_val, vx_w_idx=(0,),
                 vx_w_val=(0,), vy_w_idx=(0,), vy_w_val=(0,), **_):
        T1, T2 = _types(precision)
        if not (len(vx_s_idx) == len(vx_s_val) and len(vy_s_idx) == len(vy_s_val) and
                len(vx_w_idx) == len(vx_w_val) and len(vy_w_idx) == len(vy_w_val)):
            raise ValueError("The length of vx_s_idx, vx_s_val, vy_s_idx, vy_s_val, vx_w_idx, vx_w_val, "
                             "vy_w_idx, vy_w_val should be the same.")
        self.vx_s_idx = np.asarray(vx_s_idx).astype(T1)
        self.vx_s_val = np.asarray(vx_s_val, T2)
        self.vy_s_idx = np.asarray(vy_s_idx).astype(T1)
        self.vy_s_val = np.asarray(vy_s_val, T2)
        # water velocity BC (boundary.jl:54-68; [0] = none)
        self.vx_w_idx = np.asarray(vx_w_idx).astype(T1)
        self.vx_w_val = np.asarray(vx_w_val, T2)
        self.vy_w_idx = np.asarray(vy_w_idx).astype(T1)
        self.vy_w_val = np.asarray(vy_w_val, T2)


class VBoundary3D(VBoundary):
    dim = 3

    def __init__(self, *, precision="FP64", vx_s_idx, vx_s_val, vy_s_idx, vy_s_val, vz_s_idx,
                 vz_s_val, vx_w_idx=(0,), vx_w_val=(0,), vy_w_idx=(0,), vy_w_val=(0,), vz_w_idx=(0,),
                 vz_w_val=(0,), **_):
        T1, T2 = _types(precision)
        if not (len(vx_s_idx) == len(vx_s_val) and len(vy_s_idx) == len(vy_s_val)
                and len(vz_s_idx) == len(vz_s_val) and len(vx_w_idx) == len(vx_w_val)
                and len(vy_w_idx) == len(vy_w_val) and len(vz_w_idx) == len(vz_w_val)):
            raise ValueError("The length of vx_s_idx, vx_s_val, vy_s_idx, vy_s_val, vz_s_idx, "
                             "vz_s_val (and the water BC arrays) should be the same.")
        water = {"x": (vx_w_idx, vx_w_val), "y": (vy_w_idx, vy_w_val), "z": (vz_w_idx, vz_w_val)}
        for c, (idx, val) in water.items():
            setattr(self, f"v{c}_w_idx", np.asarray(idx).astype(T1))
            setattr(self, f"v{c}_w_val", np.asarray(val, T2))
        self.vx_s_idx = np.asarray(vx_s_idx).astype(T1)
        self.vx_s_val = np.asarray(vx_s_val, T2)
        self.vy_s_idx = np.asarray(vy_s_idx).astype(T1)
        self.vy_s_val = np.asarray(vy_s_val, T2)
        self.vz_s_idx = np.asarray(vz_s_idx).astype(T1)
        self.vz_s_val = np.asarray(vz_s_val, T2)


def UserVBoundary2D(*, ϵ="FP64", **kw):
    kw = _norm_kwargs(kw)
    return VBoundary2D(precision=kw.pop("precision", ϵ), **kw)


def UserVBoundary3D(*, ϵ="FP64", **kw):
    kw = _norm_kwargs(kw)
    return VBoundary3D(precision=kw.pop("precision", ϵ), **kw)


# ---------------------------------------------------------------------------
# meshbuilder (src/toolkits/meshbuilder.jl:16-37): particle lattice, y fastest.
# ---------------------------------------------------------------------------
def meshbuilder(x, y, z=None):
    x = np.asarray(x, np.float64)
    y = np.asarray(y, np.float64)
    if z is None:
        X = np.repeat(x, len(y))
        Y = np.tile(y, len(x))
        return np.stack([X, Y], axis=1)
    z = np.asarray(z, np.float64)
    Z, X, Y = np.meshgrid(z, x, y, indexing="ij")
    return np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)


def jl_range(a, step, b):
    """Values of the Julia range a:step:b."""
    return _axis(a, b, step)
