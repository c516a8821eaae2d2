"""The C ABI (include/mpm_b200.h) without a GPU: the library loads, exports
every entry point the header declares, its struct layouts match both a C
compiler's reading of the header and the ctypes binding, and descriptor
validation rejects bad input before touching the device."""
import ctypes as C
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "mpm_b200.h")


@pytest.fixture(scope="module")
def L(pkg):
    pkg._lib.build()
    return pkg._lib.lib()


def header_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^[A-Za-z_][\w \*]*?\b(mpm_\w+)\s*\(", text, flags=re.M)))


def header_defines():
    out = {}
    for name, val in re.findall(r"^#define (MPM_\w+)\s+(.+?)\s*(?:/\*.*)?$", open(HEADER).read(), flags=re.M):
        val = val.strip()
        if val.endswith("\\") or not val:
            continue
        try:
            out[name] = eval(val.replace("1u", "1"), {})
        except Exception:
            pass
    return out


def test_header_declares_the_binding_exports(pkg):
    assert header_functions() == sorted(pkg._lib.EXPORTS)


def test_library_exports_every_header_symbol(L):
    for name in header_functions():
        assert hasattr(L, name), name


def test_constants_match_header(pkg):
    d = header_defines()
    lib = pkg._lib
    assert d["MPM_ABI_VERSION"] == lib.ABI_VERSION
    for code, name in lib.ERRORS.items():
        assert d[name] == code
    for k in ("LINEARELASTIC", "DRUCKERPRAGER", "MOHRCOULOMB"):
        assert d["MPM_" + k] == getattr(lib, k)
    assert d["MPM_PREC_MIXED"] == lib.PREC_MIXED and d["MPM_PREC_FP64"] == lib.PREC_FP64
    for k in ("T_F64", "T_F32", "T_I64", "T_I32"):
        assert d["MPM_" + k] == getattr(lib, k)
    for k in ("XI", "VS", "SIG", "EPS", "EPSQ", "EPSK", "EPSV", "OMEGA", "MS", "SIGM", "F", "RHO", "P2C"):
        assert d["MPM_F_" + k] == getattr(lib, "F_" + k), k
    assert lib.F_REFERENCE == 0x3FF
    assert d["MPM_NOALLOC_MAX_PARTICLES"] == lib.NOALLOC_MAX_PARTICLES
    assert d["MPM_NOALLOC_MAX_KEYS"] == lib.NOALLOC_MAX_KEYS


def test_struct_layouts_match_c_compiler(pkg, tmp_path):
    """Offsets of every field as gcc lays the header out == the ctypes binding."""
    lib = pkg._lib
    structs = {"mpm_desc": lib.Desc, "mpm_view": lib.View, "mpm_host_views": lib.HostViews,
               "mpm_stats": lib.Stats}
    src = ["#include <stdio.h>", "#include <stddef.h>", '#include "mpm_b200.h"', "int main(void){"]
    for cname, py in structs.items():
        src.append(f'printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            src.append(f'printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    src.append("return 0;}")
    c = tmp_path / "layout.c"
    c.write_text("\n".join(src))
    exe = tmp_path / "layout"
    subprocess.check_call(["gcc", "-std=c99", "-I", os.path.dirname(HEADER), str(c), "-o", str(exe)])
    got = {}
    for line in subprocess.check_output([str(exe)]).decode().splitlines():
        s, f, v = line.split()
        got[(s, f)] = int(v)
    for cname, py in structs.items():
        assert got[(cname, "sizeof")] == C.sizeof(py), cname
        for f, _ in py._fields_:
            assert got[(cname, f)] == getattr(py, f).offset, (cname, f)


def test_abi_sizes_entry_point(pkg, L):
    lib = pkg._lib
    s = [C.c_int64() for _ in range(4)]
    assert L.mpm_abi_sizes(*[C.byref(x) for x in s]) == 0
    assert [x.value for x in s] == [C.sizeof(lib.Desc), C.sizeof(lib.View), C.sizeof(lib.HostViews),
                                    C.sizeof(lib.Stats)]


def _desc(pkg, **over):
    case = pkg.workloads.column_collapse_3d(h=0.04, column=(0.08, 0.08, 0.08), domain=(0.16, 0.12, 0.12))
    d = pkg.solver.make_desc(case.args, case.grid, case.mp, case.attr)
    for k, v in over.items():
        setattr(d, k, v)
    return d


@pytest.mark.parametrize("over,code,msg", [
    (dict(abi_version=99), -1, b"ABI version"),
    (dict(dim=4), -1, b"dim"),
    (dict(np=-1), -1, b"np"),
    (dict(nmat=0), -1, b"material"),
    (dict(nnx=3), -1, b"4 nodes"),
    (dict(dx=0.0), -1, b"cell size"),
    (dict(lpx=0.05), -1, b"particle size"),      # lp > h: more than 3 uGIMP nodes per axis
    (dict(constitutive=3), -8, b"constitutive"),
    (dict(mc3d=5), -1, b"mc3d"),
])
def test_create_rejects_bad_descriptors(pkg, L, over, code, msg):
    """Validation runs before any CUDA call, so it is exercised without a GPU."""
    h = C.c_void_p(123)
    rc = L.mpm_create(C.byref(_desc(pkg, **over)), C.byref(h))
    assert rc == code
    assert h.value is None
    assert msg in L.mpm_last_error(None)


def test_null_arguments(L):
    h = C.c_void_p()
    assert L.mpm_create(None, C.byref(h)) == -1
    assert L.mpm_step(None, 1e-4, 0.0, 1, None) != 0
    assert L.mpm_destroy(None) in (0, -1)


def test_product_path_fails_loudly_without_a_device(pkg):
    """No CPU fallback: without a usable GPU, host2device raises."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    case = pkg.workloads.column_collapse_3d(h=0.04, column=(0.08, 0.08, 0.08), domain=(0.16, 0.12, 0.12))
    with pytest.raises(pkg._lib.MPMError) as e:
        pkg.DeviceModel(case.args, case.grid, case.mp, case.attr, case.bc)
    assert e.value.code == -2
