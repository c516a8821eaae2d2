"""ctypes binding of libmpm_b200.so (C ABI declared in include/mpm_b200.h).

The shared library is built in-tree (``materialpointsolver.jl_b200/libmpm_b200.so``)
by ``build()``.  Loading fails loudly when it is missing: there is no CPU
fallback for the device step.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmpm_b200.so")
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ABI_VERSION = 1

MPM_OK = 0
ERRORS = {
    -1: "MPM_E_ARG", -2: "MPM_E_CUDA", -3: "MPM_E_OUT_OF_GRID", -4: "MPM_E_NONPOSITIVE_J",
    -5: "MPM_E_NAN", -6: "MPM_E_STATE", -7: "MPM_E_CELL_OVERFLOW", -8: "MPM_E_UNSUPPORTED",
}
LINEARELASTIC, DRUCKERPRAGER, MOHRCOULOMB = 0, 1, 2
PREC_MIXED, PREC_FP64 = 0, 1
SCHEME_MUSL, SCHEME_USL = 0, 1
COUPLING_OS, COUPLING_TS = 0, 1
T_F64, T_F32, T_I64, T_I32 = 0, 1, 2, 3

F_XI, F_VS, F_SIG, F_EPS, F_EPSQ, F_EPSK, F_EPSV = (1 << i for i in range(7))
F_OMEGA, F_MS, F_SIGM, F_F, F_RHO, F_P2C = (1 << i for i in range(7, 13))
F_MW, F_VW, F_SIGW, F_EPSW, F_N, F_RHOW = (1 << i for i in range(13, 19))
F_REFERENCE = F_SIGM | F_VS | F_XI | F_OMEGA | F_SIG | F_EPSK | F_EPSQ | F_EPSV | F_EPS | F_MS
F_REFERENCE_TS = F_REFERENCE | F_MW | F_VW | F_SIGW | F_EPSW | F_N
F_SNAPSHOT = F_SIG | F_EPS | F_EPSQ | F_EPSK | F_EPSV | F_XI | F_VS | F_OMEGA | F_MS
F_SNAPSHOT_TS = F_SNAPSHOT | F_SIGW | F_EPSW | F_VW | F_N

EXPORTS = [
    "mpm_create", "mpm_upload", "mpm_destroy", "mpm_step", "mpm_step_async", "mpm_sync",
    "mpm_download", "mpm_compute_p2c", "mpm_download_order", "mpm_sort", "mpm_run_stages",
    "mpm_download_grid", "mpm_get_stats", "mpm_last_error", "mpm_peak_bandwidth",
    "mpm_set_profiling", "mpm_get_kernel_times", "mpm_abi_sizes", "mpm_cell_order_noalloc",
    "mpm_grf_eval", "mpm_set_tuning", "mpm_get_tuning", "mpm_set_tile", "mpm_get_tile", "mpm_autotune",
    "mpm_mlp_nparams", "mpm_mlp_forward", "mpm_mlp_grad", "mpm_mlp_adam", "mpm_set_surrogate", "mpm_log_samples",
    "mpm_h5_create", "mpm_h5_write", "mpm_h5_close", "mpm_snapshot", "mpm_snapshot_wait",
]
NOALLOC_MAX_PARTICLES = 1 << 19
NOALLOC_MAX_KEYS = 1 << 19


class Desc(C.Structure):
    _fields_ = [
        ("abi_version", C.c_int32), ("dim", C.c_int32), ("precision", C.c_int32), ("device", C.c_int32),
        ("np", C.c_int64), ("nmat", C.c_int64),
        ("nnx", C.c_int64), ("nny", C.c_int64), ("nnz", C.c_int64),
        ("x1", C.c_double), ("y1", C.c_double), ("z1", C.c_double),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
        ("lpx", C.c_double), ("lpy", C.c_double), ("lpz", C.c_double),
        ("constitutive", C.c_int32), ("va", C.c_int32), ("mvl", C.c_int32), ("mc3d", C.c_int32),
        ("FLIP", C.c_double), ("PIC", C.c_double), ("zeta_s", C.c_double), ("gravity", C.c_double),
        ("Te", C.c_double),
        ("time_f32", C.c_int32), ("sort_every", C.c_int32), ("scheme", C.c_int32), ("coupling", C.c_int32),
        ("zeta_w", C.c_double),
    ]


class View(C.Structure):
    _fields_ = [("ptr", C.c_void_p), ("type", C.c_int32), ("pad", C.c_int32), ("ld", C.c_int64)]


_VIEW_NAMES = ["xi", "vs", "sig", "eps", "epsq", "epsk", "epsv", "Omega", "Omega0", "rho", "rho0",
               "F", "ms", "sigm", "p2c", "nid"]


class HostViews(C.Structure):
    _fields_ = ([(n, View) for n in _VIEW_NAMES] +
                [(n, View) for n in ("Ks", "Gs", "c", "phi", "psi", "sigt", "Hp", "cr")] +
                [(n, View) for n in ("vx_idx", "vx_val", "vy_idx", "vy_val", "vz_idx", "vz_val")] +
                [(n, View) for n in ("n", "rhow", "sigw", "vw", "epsw", "mw", "Kw", "kperm")] +
                [(n, View) for n in ("vxw_idx", "vxw_val", "vyw_idx", "vyw_val", "vzw_idx", "vzw_val")])


class Stats(C.Structure):
    _fields_ = [
        ("steps_done", C.c_int64), ("sorts_done", C.c_int64), ("active_nodes", C.c_int64),
        ("launches", C.c_int64),
        ("error_flags", C.c_int32), ("kernels_per_step", C.c_int32),
        ("last_step_ms", C.c_double), ("device_bytes", C.c_double),
        ("surr_rows", C.c_int64), ("surr_fallbacks", C.c_int64),
    ]


NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
              "-Xcompiler", "-fPIC", "-Xcompiler", "-fopenmp", "-shared", "-lgomp"]


TRANSLATION_UNITS = ["mpm_b200.cu", "mpm_noalloc.cu", "mpm_grf.cu", "mpm_mlp.cu", "mpm_h5.cpp"]


def sources():
    return [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC))
            if f.endswith((".cu", ".cuh", ".cpp"))] + [os.path.join(INCLUDE, "mpm_b200.h")]


def build(force=False, verbose=False):
    """Compile libmpm_b200.so for sm_100a with nvcc (in-tree)."""
    srcs = sources()
    if (not force and os.path.exists(LIB_PATH)
            and all(os.path.getmtime(LIB_PATH) >= os.path.getmtime(s) for s in srcs)):
        return LIB_PATH
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc] + NVCC_FLAGS + ["-o", LIB_PATH] + [os.path.join(CSRC, f) for f in TRANSLATION_UNITS]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    return LIB_PATH


_lib = None


def lib():
    """Load the in-tree library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with __graft_entry__.build() "
                           "(the device step has no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    L.mpm_create.argtypes = [C.POINTER(Desc), C.POINTER(vp)]
    L.mpm_upload.argtypes = [vp, C.POINTER(HostViews)]
    L.mpm_destroy.argtypes = [vp]
    L.mpm_step.argtypes = [vp, C.c_double, C.c_double, C.c_int64, C.POINTER(C.c_double)]
    L.mpm_step_async.argtypes = [vp, C.c_double, C.c_double, C.c_int64]
    L.mpm_sync.argtypes = [vp]
    L.mpm_download.argtypes = [vp, C.POINTER(HostViews), C.c_uint32]
    L.mpm_compute_p2c.argtypes = [vp, C.POINTER(C.c_int64)]
    L.mpm_download_order.argtypes = [vp, C.POINTER(C.c_int64)]
    L.mpm_sort.argtypes = [vp]
    L.mpm_run_stages.argtypes = [vp, C.c_double, C.c_double, C.c_uint32]
    L.mpm_download_grid.argtypes = [vp, C.c_int32, C.POINTER(C.c_double)]
    L.mpm_get_stats.argtypes = [vp, C.POINTER(Stats)]
    L.mpm_last_error.argtypes = [vp]
    L.mpm_last_error.restype = C.c_char_p
    L.mpm_peak_bandwidth.argtypes = [C.c_int32, C.POINTER(C.c_double)]
    L.mpm_set_profiling.argtypes = [vp, C.c_int32]
    L.mpm_get_kernel_times.argtypes = [vp, C.POINTER(C.c_char_p), C.POINTER(C.c_double),
                                       C.POINTER(C.c_int64), C.c_int32, C.POINTER(C.c_int32)]
    L.mpm_abi_sizes.argtypes = [C.POINTER(C.c_int64)] * 4
    L.mpm_cell_order_noalloc.argtypes = [C.POINTER(Desc)] + [C.c_void_p] * 6
    L.mpm_set_tuning.argtypes = [vp, C.c_int32, C.c_int32]
    L.mpm_get_tuning.argtypes = [vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
    L.mpm_set_tile.argtypes = [vp, C.c_int32, C.c_int32, C.c_int32]
    L.mpm_get_tile.argtypes = [vp] + [C.POINTER(C.c_int32)] * 3
    L.mpm_autotune.argtypes = [vp, C.c_double, C.c_double, C.c_int64, C.POINTER(C.c_double),
                               C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_double), C.c_int32]
    L.mpm_set_surrogate.argtypes = [vp, vp, vp, C.c_int32, C.c_float, C.c_float, C.c_int32]
    L.mpm_log_samples.argtypes = [vp, vp, vp, vp, C.c_uint32, C.c_uint32]
    L.mpm_mlp_nparams.argtypes = []
    L.mpm_mlp_forward.argtypes = [vp, vp, vp, vp, C.c_int64, C.c_int32, vp, vp]
    L.mpm_mlp_grad.argtypes = [vp, vp, vp, vp, C.c_int64, C.c_float, C.c_int32, vp, vp, vp, vp]
    L.mpm_mlp_adam.argtypes = [vp, vp, vp, vp, C.c_float, C.c_float, C.c_float, C.c_float, C.c_int64, vp]
    L.mpm_grf_eval.argtypes = [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64,
                               C.c_double, C.c_void_p]
    L.mpm_h5_create.argtypes = [C.c_char_p, C.POINTER(vp)]
    L.mpm_h5_write.argtypes = [vp, C.c_char_p, C.c_int32, C.c_int32, C.POINTER(C.c_int64), vp]
    L.mpm_h5_close.argtypes = [vp]
    L.mpm_snapshot.argtypes = [vp, vp, C.c_int64, C.c_double, C.c_uint32, C.c_int32]
    L.mpm_snapshot_wait.argtypes = [vp, C.POINTER(C.c_int64)]
    sizes = [C.c_int64() for _ in range(4)]
    L.mpm_abi_sizes(*[C.byref(x) for x in sizes])
    mine = [C.sizeof(Desc), C.sizeof(View), C.sizeof(HostViews), C.sizeof(Stats)]
    if [x.value for x in sizes] != mine:
        raise RuntimeError(f"C ABI struct sizes {[x.value for x in sizes]} != binding {mine}")
    _lib = L
    return L


class MPMError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


def check(rc, handle=None):
    if rc != MPM_OK:
        msg = lib().mpm_last_error(handle)
        raise MPMError(rc, msg.decode() if msg else "")
    return rc
