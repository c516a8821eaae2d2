"""mpm_cell_order_noalloc: the allocation-free cell ordering.

Callers that cannot allocate device memory (a host runtime with its own
device-memory pool, real-time loops that must not hit the allocator's implicit
synchronisation) pass their own device buffers and get the particle-to-cell indices and the
cell-sorted particle order; the entry point uses a fixed static scratch area
instead of cudaMalloc.  Its output must equal what the allocating path
(mpm_compute_p2c, mpm_sort + mpm_download_order) returns for the same
positions -- integer results, so compared exactly -- on two calls in a row,
since every call reuses the scratch left behind by the previous one.

This file is named to be collected last, so that a failure here comes after
every other test has already run.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _case(pkg, dim, dense=False):
    if dense:
        # more than 32 particles in each of more than 4096 cells: every cell's
        # bucket goes through the queue of large buckets and the CTA sort
        if dim == 2:   # 6 x 6 per cell, 100 x 50 cells: 180 000 particles
            return pkg.workloads.column_collapse_2d(h=0.01, ppc=6, width=1.0, height=0.5, domain=(1.2, 0.6),
                                                    seed=23)
        # 4 x 4 x 4 per cell, 20 x 12 x 20 cells: 307 200 particles
        return pkg.workloads.column_collapse_3d(h=0.01, ppc=4, column=(0.2, 0.12, 0.2), domain=(0.24, 0.16, 0.24),
                                                seed=24)
    if dim == 2:
        return pkg.workloads.column_collapse_2d(h=0.01, width=0.1, height=0.06, domain=(0.2, 0.1), seed=21)
    return pkg.workloads.column_collapse_3d(h=0.02, column=(0.12, 0.08, 0.12), domain=(0.24, 0.12, 0.16),
                                            seed=22)


@pytest.mark.parametrize("dense", [False, True])
@pytest.mark.parametrize("dim", [2, 3])
def test_noalloc_matches_allocating_path(pkg, gpu_lib, dim, dense):
    import torch

    case = _case(pkg, dim, dense)
    if dense:
        big = np.bincount(_cells(case, dim)) > 32
        assert big.sum() > 4096
    rng = np.random.default_rng(40 + dim)
    # shuffle the particles so the ordering has real work to do
    case.mp.xi[:] = case.mp.xi[rng.permutation(case.mp.np)]

    dev = pkg.DeviceModel(case.args, case.grid, case.mp, case.attr, case.bc)
    p2c_ref = dev.p2c()
    dev.sort()
    order_ref = dev.order()
    desc = pkg.solver.make_desc(case.args, case.grid, case.mp, case.attr)
    dev.close()

    npart = case.mp.np
    cols = [torch.tensor(np.ascontiguousarray(case.mp.xi[:, d]), dtype=torch.float64, device="cuda")
            for d in range(dim)]
    z = cols[2] if dim == 3 else cols[0]
    for call in range(2):
        order = torch.full((npart,), -7, dtype=torch.int64, device="cuda")
        p2c = torch.full((npart,), -7, dtype=torch.int64, device="cuda")
        rc = gpu_lib.mpm_cell_order_noalloc(C.byref(desc), cols[0].data_ptr(), cols[1].data_ptr(), z.data_ptr(),
                                            order.data_ptr(), p2c.data_ptr(), None)
        assert rc == 0, gpu_lib.mpm_last_error(None)
        assert np.array_equal(p2c.cpu().numpy(), p2c_ref), f"p2c differs on call {call}"
        assert np.array_equal(order.cpu().numpy(), order_ref), f"order differs on call {call}"


def _cells(case, dim):
    g = case.grid
    lo = [g.x1, g.y1, g.z1 if dim == 3 else 0.0]
    h = [g.dx, g.dy, g.dz if dim == 3 else 1.0]
    c = [np.floor((case.mp.xi[:, d] - lo[d]) / h[d]).astype(np.int64) for d in range(dim)]
    return c[0] * 1000 + c[1] if dim == 2 else (c[2] * 1000 + c[0]) * 1000 + c[1]


def test_noalloc_rejects_oversize(pkg, gpu_lib):
    case = _case(pkg, 3)
    desc = pkg.solver.make_desc(case.args, case.grid, case.mp, case.attr)
    desc.np = pkg._lib.NOALLOC_MAX_PARTICLES + 1
    dummy = C.c_void_p(16)   # never dereferenced: the size check comes first
    rc = gpu_lib.mpm_cell_order_noalloc(C.byref(desc), dummy, dummy, dummy, dummy, dummy, None)
    assert rc == -1
    assert b"MPM_NOALLOC_MAX_PARTICLES" in gpu_lib.mpm_last_error(None)
