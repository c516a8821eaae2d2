"""Host <-> device transfers of the C ABI (mpm_upload / mpm_download, the
host2device / device2host! pair of ext/CUDAExt/devicehelpfunc_cuda.jl:17-69).

The copies are staged through the sort's spare particle buffer and issued
without per-column host synchronisation; these checks pin what that must
preserve: every field lands in the caller's arrays in the original particle
order, FP32 views receive exactly the FP32 rounding of the FP64 result (derived
fields -- Ω, σm, ρs -- included), the per-particle mass Ω·ρs formed on the
device equals the host product, and a second upload into a used handle
replaces its state."""
import numpy as np
import pytest

from helpers import fresh_particles

FIELDS = ("xi", "vs", "sig", "eps", "epsq", "epsk", "epsv", "Omega", "sigm", "ms")


def column(pkg, **kw):
    base = dict(h=0.01, Ttol=0.01, gpu_precision="mixed")
    base.update(kw)
    return pkg.workloads.column_collapse_2d(**base)


def as_precision(pkg, mp, precision):
    """An empty output struct of `mp`'s shape with host arrays of `precision`."""
    w = dict(phase=2, n=mp.n, rho_w=mp.rho_w) if getattr(mp, "phase", 1) == 2 else {}
    return pkg.Particle2D(precision=precision, dx=mp.dx, dy=mp.dy, xi=mp.xi, rho=mp.rho, **w)


@pytest.mark.gpu
@pytest.mark.parametrize("gpu_precision", ["mixed", "fp64"])
def test_fp32_views_are_the_rounded_fp64_views(pkg, gpu_lib, gpu_precision):
    c = column(pkg, gpu_precision=gpu_precision)
    dev = pkg.DeviceModel(c.args, c.grid, c.mp, c.attr, c.bc)
    try:
        dev.step(c.dt, 0.0, 40)
        o64 = as_precision(pkg, c.mp, "FP64")
        o32 = as_precision(pkg, c.mp, "FP32")
        dev.download(pkg._lib.F_REFERENCE | pkg._lib.F_RHO, o64)
        dev.download(pkg._lib.F_REFERENCE | pkg._lib.F_RHO, o32)
    finally:
        dev.close()
    for k in FIELDS + ("rho",):
        a64, a32 = getattr(o64, k), getattr(o32, k)
        assert a32.dtype == np.float32 and a64.dtype == np.float64, k
        assert np.array_equal(a32, a64.astype(np.float32)), k
    assert np.abs(o64.vs).max() > 0 and np.abs(o64.sig).max() > 0


@pytest.mark.gpu
def test_download_keeps_the_original_order_across_sorts(pkg, gpu_lib):
    """Particles re-sorted 10 times on the device come back in the caller's
    order: with no motion (no gravity, no stress) every field returns
    unchanged, per particle."""
    c = column(pkg, gravity=0.0)
    c.args.sort_every = 2
    dev = pkg.DeviceModel(c.args, c.grid, c.mp, c.attr, c.bc)
    try:
        dev.step(c.dt, 0.0, 20)
        out = fresh_particles(pkg, c.mp)
        dev.download(pkg._lib.F_REFERENCE, out)
    finally:
        dev.close()
    assert np.array_equal(out.xi, c.mp.xi)          # jittered: unique per particle
    # Ω = det(F)·Ω0 with Ω0 stored in FP32 (mixed mode) and det(F) = 1
    assert np.array_equal(out.Omega, c.mp.Omega.astype(np.float32).astype(np.float64))
    assert not out.vs.any() and not out.sig.any()


@pytest.mark.gpu
def test_device_mass_is_the_host_product(pkg, gpu_lib):
    c = column(pkg, gpu_precision="fp64")
    rng = np.random.default_rng(4)
    c.mp.rho[:] = rng.uniform(1500.0, 2500.0, c.mp.np)
    c.mp.rho0[:] = c.mp.rho
    dev = pkg.DeviceModel(c.args, c.grid, c.mp, c.attr, c.bc)
    try:
        out = fresh_particles(pkg, c.mp)
        dev.download(pkg._lib.F_MS, out)
    finally:
        dev.close()
    assert np.array_equal(out.ms, c.mp.Omega * c.mp.rho)


@pytest.mark.gpu
def test_second_upload_replaces_the_state(pkg, gpu_lib):
    """mpm_upload into a handle that has stepped (and sorted) restarts it from
    the new host arrays: stepping again matches a fresh handle to the
    run-to-run spread of the FP32 reductions."""
    c = column(pkg)
    dev = pkg.DeviceModel(c.args, c.grid, c.mp, c.attr, c.bc)
    try:
        dev.step(c.dt, 0.0, 50)
        dev.upload()                       # the unchanged initial host arrays
        dev.step(c.dt, 0.0, 30)
        a = fresh_particles(pkg, c.mp)
        dev.download(pkg._lib.F_REFERENCE, a)
    finally:
        dev.close()
    dev = pkg.DeviceModel(c.args, c.grid, c.mp, c.attr, c.bc)
    try:
        dev.step(c.dt, 0.0, 30)
        b = fresh_particles(pkg, c.mp)
        dev.download(pkg._lib.F_REFERENCE, b)
    finally:
        dev.close()
    da, db = a.xi - c.mp.xi, b.xi - c.mp.xi
    assert np.linalg.norm(da - db) <= 1e-4 * np.linalg.norm(db)
    assert np.linalg.norm(db) > 0
