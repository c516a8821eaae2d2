"""ctypes binding of the FP64 CPU oracle (oracle/mpm_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, bench.py's CPU-baseline and
reference legs, and __graft_entry__.smoke() as the checker.  The product
package never imports this module.

The oracle restates MaterialPointSolver.jl's CPU path for the OS/MUSL uGIMP
step; its parity with the reference is UNPINNED (no runnable Julia and no
golden vectors in the reference's tests) and is cross-checked by hand-derived
known-answer tests and an independent pure-Python transliteration.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int64)


class OrcModel(C.Structure):
    _fields_ = [
        ("dim", C.c_int32), ("nic", C.c_int32),
        ("nnx", C.c_int64), ("nny", C.c_int64), ("nnz", C.c_int64),
        ("ncx", C.c_int64), ("ncy", C.c_int64), ("ncz", C.c_int64),
        ("ni", C.c_int64), ("nc", C.c_int64),
        ("x1", C.c_double), ("y1", C.c_double), ("z1", C.c_double),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
        ("g_xi", _dp), ("g_ms", _dp),
        ("g_ps", _dp), ("g_fs", _dp), ("g_vs", _dp), ("g_vsT", _dp), ("g_as", _dp), ("g_dus", _dp),
        ("g_sigm", _dp), ("g_omega", _dp),
        ("np", C.c_int64),
        ("lpx", C.c_double), ("lpy", C.c_double), ("lpz", C.c_double),
        ("p2c", _ip), ("p2n", _ip),
        ("Nij", _dp), ("dNx", _dp), ("dNy", _dp), ("dNz", _dp),
        ("xi", _dp), ("vs", _dp), ("ps", _dp),
        ("ms", _dp), ("Omega", _dp), ("Omega0", _dp), ("rho", _dp), ("rho0", _dp),
        ("sig", _dp), ("eps", _dp), ("deps", _dp), ("sij", _dp),
        ("sigm", _dp), ("epsq", _dp), ("epsk", _dp), ("epsv", _dp),
        ("dF", _dp), ("F", _dp),
        ("nid", _ip),
        ("Ks", _dp), ("Gs", _dp), ("c", _dp), ("phi", _dp), ("psi", _dp), ("sigt", _dp),
        ("Hp", _dp), ("cr", _dp),
        ("vx_idx", _ip), ("vy_idx", _ip), ("vz_idx", _ip),
        ("vx_val", _dp), ("vy_val", _dp), ("vz_val", _dp),
        ("Te", C.c_double), ("gravity", C.c_double), ("FLIP", C.c_double), ("PIC", C.c_double),
        ("zeta_s", C.c_double),
        ("constitutive", C.c_int32), ("va", C.c_int32), ("mvl", C.c_int32), ("mc3d", C.c_int32),
        ("nthreads", C.c_int32), ("scheme", C.c_int32),
        ("coupling", C.c_int32), ("f32", C.c_int32), ("zeta_w", C.c_double),
        ("g_mi", _dp), ("g_mw", _dp),
        ("g_pw", _dp), ("g_fw", _dp), ("g_fd", _dp), ("g_vw", _dp), ("g_vwT", _dp), ("g_aw", _dp),
        ("g_duw", _dp),
        ("mw", _dp), ("mi", _dp), ("n", _dp), ("rhow", _dp), ("rhow0", _dp), ("sigw", _dp),
        ("vw", _dp), ("pw", _dp), ("epsw", _dp), ("depsw", _dp),
        ("Kw", _dp), ("kperm", _dp),
        ("vxw_idx", _ip), ("vyw_idx", _ip), ("vzw_idx", _ip),
        ("vxw_val", _dp), ("vyw_val", _dp), ("vzw_val", _dp),
    ]


CONSTITUTIVE = {"linearelastic": 0, "druckerprager": 1, "mohrcoulomb": 2}


def build(force=False):
    """Compile the oracle with g++ (OpenMP) into oracle/_build/liboracle.so."""
    os.makedirs(os.path.join(HERE, "_build"), exist_ok=True)
    src = os.path.join(HERE, "mpm_oracle.cpp")
    if (not force and os.path.exists(LIB_PATH)
            and os.path.getmtime(LIB_PATH) >= os.path.getmtime(src)
            and os.path.getmtime(LIB_PATH) >= os.path.getmtime(os.path.join(HERE, "mpm_oracle.h"))):
        return LIB_PATH
    cmd = ["g++", "-O2", "-fopenmp", "-fPIC", "-shared", "-std=c++17", "-ffp-contract=off",
           "-o", LIB_PATH, src]
    subprocess.check_call(cmd)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        L.orc_procedure.argtypes = [C.POINTER(OrcModel), C.c_double, C.c_double]
        L.orc_run.argtypes = [C.POINTER(OrcModel), C.c_double, C.c_double, C.c_int64, _dp]
        L.orc_fld.restype = C.c_double
        L.orc_fld.argtypes = [C.c_double, C.c_double]
        L.orc_cld.restype = C.c_double
        L.orc_cld.argtypes = [C.c_double, C.c_double]
        L.orc_p2c.argtypes = [C.POINTER(OrcModel), _dp, C.c_int64, _ip]
        L.orc_ugimp.argtypes = [C.c_double, C.c_double, C.c_double, _dp, _dp]
        L.orc_dp_point.argtypes = [C.c_int, _dp, _dp, _dp] + [C.c_double] * 6
        L.orc_mc3d_point.argtypes = [_dp, _dp, _dp, _dp] + [C.c_double] * 6
        L.orc_mc3d_yield.argtypes = [_dp, C.c_double, C.c_double, C.c_double, _dp, _dp]
        L.orc_mc3d_yield.restype = C.c_int
        for name in ("orc_resetgrid", "orc_resetmp"):
            getattr(L, name).argtypes = [C.POINTER(OrcModel)]
        L.orc_p2g.argtypes = [C.POINTER(OrcModel), C.c_double]
        L.orc_solvegrid.argtypes = [C.POINTER(OrcModel), C.c_double]
        L.orc_dm1.argtypes = [C.POINTER(OrcModel), C.c_double]
        L.orc_dm2.argtypes = [C.POINTER(OrcModel)]
        L.orc_dm3.argtypes = [C.POINTER(OrcModel), C.c_double]
        L.orc_g2p.argtypes = [C.POINTER(OrcModel), C.c_double]
        L.orc_constitutive.argtypes = [C.POINTER(OrcModel), C.c_double]
        L.orc_resetmp_ts.argtypes = [C.POINTER(OrcModel)]
        L.orc_p2g_ts.argtypes = [C.POINTER(OrcModel), C.c_double]
        L.orc_solvegrid_ts.argtypes = [C.POINTER(OrcModel), C.c_double]
        L.orc_dm1_ts.argtypes = [C.POINTER(OrcModel), C.c_double]
        L.orc_dm2_ts.argtypes = [C.POINTER(OrcModel)]
        L.orc_dm3_ts.argtypes = [C.POINTER(OrcModel), C.c_double]
        L.orc_g2p_ts.argtypes = [C.POINTER(OrcModel), C.c_double]
        _lib = L
    return _lib


def _d(a):
    return np.asfortranarray(np.asarray(a, dtype=np.float64)).copy(order="F")


def _i(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int64)).copy()


def _ptr(a, t=_dp):
    return a.ctypes.data_as(t)


class Oracle:
    """FP64 oracle state built from the host structs (copies everything)."""

    def __init__(self, args, grid, mp, attr, bc, nthreads=0):
        D = grid.dim
        self.D = D
        self.np_ = mp.np
        nv = 4 if D == 2 else 6
        ni, npart, NIC = grid.ni, mp.np, mp.NIC
        self.nthreads = nthreads
        keep = {}
        keep["g_xi"] = _d(grid.xi)
        for k in ("g_ms",):
            keep[k] = np.zeros(ni)
        for k in ("g_ps", "g_fs", "g_vs", "g_vsT", "g_as", "g_dus"):
            keep[k] = np.zeros((ni, D), order="F")
        keep["g_sigm"] = np.zeros(grid.nc)
        keep["g_omega"] = np.zeros(grid.nc)
        keep["p2c"] = np.zeros(npart, np.int64)
        keep["p2n"] = np.zeros((npart, NIC), np.int64, order="F")
        for k in ("Nij", "dNx", "dNy", "dNz"):
            keep[k] = np.zeros((npart, NIC), order="F")
        keep["xi"] = _d(mp.xi)
        keep["vs"] = _d(mp.vs)
        keep["ps"] = _d(mp.ps)
        for k in ("ms", "Omega", "Omega0", "rho", "rho0", "sigm", "epsq", "epsk", "epsv"):
            keep[k] = _d(getattr(mp, k))
        for k in ("sig", "eps", "deps", "sij", "dF", "F"):
            keep[k] = _d(getattr(mp, k))
        keep["nid"] = _i(attr.nid)
        for k in ("Ks", "Gs", "c", "phi", "psi", "sigt", "Hp", "cr"):
            keep[k] = _d(getattr(attr, k))
        zeros_i = np.zeros(ni, np.int64)
        zeros_d = np.zeros(ni)
        keep["vx_idx"] = _i(bc.vx_s_idx)
        keep["vy_idx"] = _i(bc.vy_s_idx)
        keep["vz_idx"] = _i(bc.vz_s_idx) if D == 3 else zeros_i
        keep["vx_val"] = _d(bc.vx_s_val)
        keep["vy_val"] = _d(bc.vy_s_val)
        keep["vz_val"] = _d(bc.vz_s_val) if D == 3 else zeros_d
        ts = getattr(args, "coupling", "OS") == "TS"
        if ts:
            # two-phase state (particle.jl:103-128, grid.jl TS arrays, boundary.jl water BC)
            keep["g_mi"], keep["g_mw"] = np.zeros(ni), np.zeros(ni)
            for k in ("g_pw", "g_fw", "g_fd", "g_vw", "g_vwT", "g_aw", "g_duw"):
                keep[k] = np.zeros((ni, D), order="F")
            keep["mw"], keep["mi"] = np.zeros(npart), np.zeros(npart)
            keep["n"], keep["rhow"], keep["rhow0"] = _d(mp.n), _d(mp.rho_w), _d(mp.rho_w0)
            keep["sigw"] = _d(mp.sigw)
            keep["vw"] = _d(mp.vw)
            keep["pw"] = np.zeros((npart, D), order="F")
            keep["epsw"], keep["depsw"] = _d(mp.epsw), _d(mp.depsw)
            keep["Kw"] = _d(np.broadcast_to(attr.Kw, (len(attr.Es),)))
            keep["kperm"] = _d(np.broadcast_to(attr.k, (len(attr.Es),)))
            for c in "xyz":
                idx = getattr(bc, f"v{c}_w_idx", None) if (c != "z" or D == 3) else None
                full = idx is not None and len(idx) == ni
                keep[f"v{c}w_idx"] = _i(idx) if full else zeros_i
                keep[f"v{c}w_val"] = _d(getattr(bc, f"v{c}_w_val")) if full else zeros_d
        self.a = keep
        m = OrcModel()
        m.dim, m.nic = D, NIC
        m.nnx, m.nny = grid.nnx, grid.nny
        m.nnz = grid.nnz if D == 3 else 1
        m.ncx, m.ncy = grid.ncx, grid.ncy
        m.ncz = grid.ncz if D == 3 else 1
        m.ni, m.nc = ni, grid.nc
        m.x1, m.y1, m.dx, m.dy = grid.x1, grid.y1, grid.dx, grid.dy
        m.z1 = grid.z1 if D == 3 else 0.0
        m.dz = grid.dz if D == 3 else 1.0
        m.np = npart
        m.lpx, m.lpy = mp.dx, mp.dy
        m.lpz = mp.dz if D == 3 else 1.0
        for name, _t in OrcModel._fields_:
            if name in keep:
                t = _ip if keep[name].dtype == np.int64 else _dp
                setattr(m, name, _ptr(keep[name], t))
        m.Te, m.gravity, m.FLIP, m.PIC, m.zeta_s = args.Te, args.gravity, args.FLIP, args.PIC, args.zeta_s
        m.constitutive = CONSTITUTIVE[args.constitutive]
        m.va = 0 if args.va == "a" else 1
        m.mvl = int(args.MVL)
        m.mc3d = 1 if getattr(args, "mc3d", "literal") == "restated" else 0
        m.nthreads = nthreads
        m.scheme = 1 if getattr(args, "scheme", "MUSL") == "USL" else 0
        m.coupling = 1 if ts else 0
        m.zeta_w = getattr(args, "zeta_w", 0.0)
        m.f32 = 1 if getattr(args, "precision", "FP64") == "FP32" else 0
        self.m = m

    def __getattr__(self, name):
        a = self.__dict__.get("a")
        if a is not None and name in a:
            return a[name]
        raise AttributeError(name)

    def procedure(self, dt, Ti):
        return lib().orc_procedure(C.byref(self.m), dt, Ti)

    def run(self, dt, Ti0, nsteps):
        out = C.c_double(0.0)
        rc = lib().orc_run(C.byref(self.m), dt, Ti0, nsteps, C.byref(out))
        if rc:
            raise RuntimeError(f"oracle run failed: {rc}")
        return out.value

    # per-stage entry points
    def stage(self, name, *a):
        return getattr(lib(), "orc_" + name)(C.byref(self.m), *a)

    def p2c(self, xi):
        xi = _d(xi)
        out = np.zeros(xi.shape[0], np.int64)
        lib().orc_p2c(C.byref(self.m), _ptr(xi), xi.shape[0], _ptr(out, _ip))
        return out


def fld(a, b):
    return lib().orc_fld(a, b)


def cld(a, b):
    return lib().orc_cld(a, b)


def ugimp(d, h, lp):
    N, dN = C.c_double(), C.c_double()
    lib().orc_ugimp(d, h, lp, C.byref(N), C.byref(dN))
    return N.value, dN.value


def dp_point(dim, sig, epsq, epsk, K, G, c, phi, psi, sigt):
    s = np.array(sig, np.float64)
    q, k = C.c_double(epsq), C.c_double(epsk)
    lib().orc_dp_point(dim, _ptr(s), C.byref(q), C.byref(k), K, G, c, phi, psi, sigt)
    return s, q.value, k.value


def mc3d_point(sig, sig0, de, epsq, K, G, c, phi, psi, sigt):
    s = np.array(sig, np.float64)
    s0 = np.array(sig0, np.float64)
    d = np.array(de, np.float64)
    q = C.c_double(epsq)
    lib().orc_mc3d_point(_ptr(s), _ptr(s0), _ptr(d), C.byref(q), K, G, c, phi, psi, sigt)
    return s, q.value


def mc3d_yield(sig, c, phi, psi, sigt):
    """Restated 3D Mohr-Coulomb yield functions (ft, fs) of a Voigt stress."""
    s = np.array(sig, np.float64)
    ft, fs = C.c_double(), C.c_double()
    lib().orc_mc3d_yield(_ptr(s), c, phi, sigt, C.byref(ft), C.byref(fs))
    return ft.value, fs.value

