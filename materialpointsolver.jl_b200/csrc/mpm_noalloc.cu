// mpm_noalloc.cu -- the cell ordering of mpm_sort() for callers that cannot
// allocate device memory.
//
// Some host environments call into this library from places where
// cudaMalloc is not available or not allowed: a host runtime that owns all
// device memory through its own pool and forbids foreign allocations, or a
// real-time loop that must not trigger the allocator's implicit
// synchronisation.  For them, mpm_cell_order_noalloc() computes the same
// particle-to-cell indices and the same cell-sorted particle order as
// mpm_sort() + mpm_download_order(), using only the caller's input and output
// buffers plus a fixed scratch area that lives in this file as a static
// device array (MPM_NOALLOC_SCRATCH_BYTES bytes on every GPU that loads the
// library, held until the process exits).
//
// Nothing here calls cudaMalloc, cudaFree or an allocating library routine.
// The call is synchronous: it reads the sort's error word back and waits for
// its stream before returning, so it must not be issued on a stream that is
// being captured into a graph.
#include "../../include/mpm_b200.h"
#include "mpm_sort.cuh"

#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>

using namespace mpm;

namespace mpm_detail {
// defined in mpm_b200.cu: the message mpm_last_error(NULL) returns
__attribute__((visibility("hidden"))) void set_global_error(const std::string &m);
}

namespace {

constexpr int64_t NA_NP = MPM_NOALLOC_MAX_PARTICLES;
constexpr int64_t NA_NK = MPM_NOALLOC_MAX_KEYS;
// cells holding more than BUCKET_SMALL particles are queued for the CTA sort;
// np <= NA_NP particles fill at most NA_NP / (BUCKET_SMALL + 1) such cells, so
// the queue (rounded up to a power of two) can never overflow
constexpr uint32_t NA_BIG_CAP = 16384;
static_assert((int64_t)NA_BIG_CAP >= NA_NP / (BUCKET_SMALL + 1) + 1, "big-bucket queue smaller than the worst case");

// scratch layout (byte offsets, each 256-byte aligned)
constexpr size_t al(size_t b) { return (b + 255) / 256 * 256; }
constexpr size_t OFF_KEYS = 0;                                           // uint32 [NA_NP]
constexpr size_t OFF_CNT = OFF_KEYS + al(4 * NA_NP);                     // uint32 [NA_NK]
constexpr size_t OFF_OFF = OFF_CNT + al(4 * NA_NK);                      // uint32 [NA_NK + 1]
constexpr size_t OFF_BSUM = OFF_OFF + al(4 * (NA_NK + 1));               // uint32 [NA_NK / 2048 + 2]
constexpr size_t OFF_PAIRS = OFF_BSUM + al(4 * (NA_NK / SCAN_CHUNK + 2)); // uint2 [NA_NP]
constexpr size_t OFF_PAIRS2 = OFF_PAIRS + al(8 * NA_NP);                 // uint2 [NA_NP]
constexpr size_t OFF_TILES = OFF_PAIRS2 + al(8 * NA_NP);                 // uint32 [NA_NK / 64]
constexpr size_t OFF_BIG = OFF_TILES + al(4 * (NA_NK / 64 + 1));         // uint32 [NA_BIG_CAP]
constexpr size_t OFF_WORDS = OFF_BIG + al(4 * NA_BIG_CAP);               // ntiles, nbig, err
constexpr size_t SCRATCH_BYTES = OFF_WORDS + 256;
static_assert(SCRATCH_BYTES <= (size_t)MPM_NOALLOC_SCRATCH_BYTES, "scratch layout exceeds the stated size");

// The scratch area.  In host code this name is only a host-side stand-in for
// the symbol, not a device address: kernels receive the address obtained with
// cudaGetSymbolAddress() below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[MPM_NOALLOC_SCRATCH_BYTES];

constexpr int MAX_DEV = 64;
unsigned char *g_scratch_ptr[MAX_DEV] = {};
std::mutex g_setup_mu;

template <int D>
__global__ void k_na_keys(const double *x, const double *y, const double *z, int64_t np, AxisC<float> ax,
                          AxisC<float> ay, AxisC<float> az, SortGeom sg, uint32_t *keys, uint32_t *cnt,
                          int64_t *p2c_out) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    const double xp = x[i], yp = y[i], zp = D == 3 ? z[i] : 0.0;
    // cell for the key: the same rule as the step kernels (Julia fld / cld)
    int cx = clampi(cell_fld<float>(xp, ax), 0, sg.ncx - 1);
    int cy = clampi(cell_cld_m1<float>(yp, ay), 0, sg.ncy - 1);
    int cz = D == 3 ? clampi(cell_fld<float>(zp, az), 0, sg.ncz - 1) : 0;
    uint32_t k = cell_key<D>(cx, cy, cz, sg);
    // sub-cell octant, the rank order inside a cell (mpm_sort.cuh)
    uint32_t o = 0;
    if (cell_offset<float>(xp, cx, ax) >= 0.5 * ax.h) o |= 1u;
    if (cell_offset<float>(yp, cy, ay) >= 0.5 * ay.h) o |= 2u;
    if (D == 3 && cell_offset<float>(zp, cz, az) >= 0.5 * az.h) o |= 4u;
    keys[i] = k | (o << OCT_SHIFT);
    atomicAdd(&cnt[k], 1u);
    // p2c, 1-based, the reference's float formula (utils_OS.jl:247-249, 380-383)
    double qy = jl_cld(yp - ay.x1, ay.h), qx = jl_fld(xp - ax.x1, ax.h);
    double v = D == 2 ? qy + qx * (double)sg.ncy
                      : qy + jl_fld(zp - az.x1, az.h) * (double)sg.ncy * (double)sg.ncx + qx * (double)sg.ncy;
    p2c_out[i] = (v >= -9.0e18 && v <= 9.0e18) ? (int64_t)trunc(v) : (int64_t)(-1);
}

__global__ void k_na_scatter(int64_t np, const uint32_t *keys, const uint32_t *off, uint32_t *cur, uint2 *pairs) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    const uint32_t kk = keys[i], k = kk & LOW29;
    uint32_t pos = off[k] + atomicAdd(&cur[k], 1u);
    pairs[pos] = make_uint2((uint32_t)i | (kk & ~LOW29), (uint32_t)i);
}

__global__ void k_na_out(int64_t np, const uint2 *pairs2, int64_t *order_out) {
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < np) order_out[k] = (int64_t)(pairs2[k].x & LOW29);
}

inline int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }

AxisC<float> axis(double x1, double h, int64_t nn) {
    AxisC<float> c{};
    c.x1 = x1;
    c.h = h;
    c.inv_h = 1.0 / h;
    c.nn = (int)nn;
    c.nc = (int)(nn > 1 ? nn - 1 : 1);
    return c;
}

int na_fail(int code, const std::string &m) {
    mpm_detail::set_global_error(m);
    return code;
}

#define NA_CK(call)                                                                        \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess) return na_fail(MPM_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

template <int D>
int run(const mpm_desc *d, const double *x, const double *y, const double *z, int64_t *order_out,
        int64_t *p2c_out, cudaStream_t st, unsigned char *S) {
    using T = Tile<D>;
    const int64_t np = d->np;
    SortGeom sg{};
    const int64_t nk = sort_geom(sg, D, d->nnx, d->nny, d->nnz, T::TX, T::TY, T::TZ);
    if (nk > NA_NK)
        return na_fail(MPM_E_ARG, "mpm_cell_order_noalloc: the grid needs " + std::to_string(nk) +
                                      " cell keys, more than MPM_NOALLOC_MAX_KEYS (" + std::to_string(NA_NK) + ")");
    const uint32_t ntile = (uint32_t)(nk / T::CPT);
    uint32_t *keys = (uint32_t *)(S + OFF_KEYS), *cnt = (uint32_t *)(S + OFF_CNT), *off = (uint32_t *)(S + OFF_OFF);
    uint32_t *bsum = (uint32_t *)(S + OFF_BSUM), *tiles = (uint32_t *)(S + OFF_TILES), *big = (uint32_t *)(S + OFF_BIG);
    uint2 *pairs = (uint2 *)(S + OFF_PAIRS), *pairs2 = (uint2 *)(S + OFF_PAIRS2);
    uint32_t *ntiles = (uint32_t *)(S + OFF_WORDS), *nbig = ntiles + 1;
    int *err = (int *)(ntiles + 2);
    // the scratch keeps the previous call's contents: clear what must start at zero
    NA_CK(cudaMemsetAsync(cnt, 0, (size_t)nk * 4, st));
    NA_CK(cudaMemsetAsync(ntiles, 0, 12, st));
    if (np == 0) return MPM_OK;
    AxisC<float> ax = axis(d->x1, d->dx, d->nnx), ay = axis(d->y1, d->dy, d->nny);
    AxisC<float> az = D == 3 ? axis(d->z1, d->dz, d->nnz) : axis(0.0, 1.0, 2);
    k_na_keys<D><<<cdiv(np, 256), 256, 0, st>>>(x, y, z, np, ax, ay, az, sg, keys, cnt, p2c_out);
    const uint32_t nb = (uint32_t)cdiv(nk, SCAN_CHUNK);
    k_scan_reduce<<<nb, SCAN_T, 0, st>>>(cnt, (uint32_t)nk, bsum);
    k_scan_top<<<1, SCAN_T, 0, st>>>(bsum, nb);
    k_scan_down<<<nb, SCAN_T, 0, st>>>(cnt, (uint32_t)nk, bsum, off);
    NA_CK(cudaMemsetAsync(cnt, 0, (size_t)nk * 4, st));
    k_na_scatter<<<cdiv(np, 256), 256, 0, st>>>(np, keys, off, cnt, pairs);
    k_sort_buckets<<<cdiv(nk, 256), 256, 0, st>>>(off, (uint32_t)nk, pairs, big, nbig, NA_BIG_CAP, err);
    k_sort_big<<<64, 512, 0, st>>>(off, big, nbig, NA_BIG_CAP, pairs);
    k_tile_list<<<cdiv(ntile, 256), 256, 0, st>>>(off, ntile, T::CPT, tiles, ntiles);
    k_tile_transpose<T::CPT><<<148 * 8, T::CPT, 0, st>>>(off, tiles, ntiles, pairs, pairs2);
    k_na_out<<<cdiv(np, 256), 256, 0, st>>>(np, pairs2, order_out);
    NA_CK(cudaGetLastError());
    int e = 0;
    NA_CK(cudaMemcpyAsync(&e, err, 4, cudaMemcpyDeviceToHost, st));
    NA_CK(cudaStreamSynchronize(st));
    if (e & ERR_OVF) return na_fail(MPM_E_CELL_OVERFLOW, "more than 4096 particles in one cell");
    return MPM_OK;
}

}  // namespace

extern "C" int mpm_cell_order_noalloc(const mpm_desc *d, const double *x, const double *y, const double *z,
                                      int64_t *order_out, int64_t *p2c_out, void *stream) {
    if (!d || !x || !y || (d && d->dim == 3 && !z) || !order_out || !p2c_out)
        return na_fail(MPM_E_ARG, "mpm_cell_order_noalloc: null argument");
    if (d->dim != 2 && d->dim != 3) return na_fail(MPM_E_ARG, "mpm_cell_order_noalloc: dim must be 2 or 3");
    if (d->np < 0 || d->np > NA_NP)
        return na_fail(MPM_E_ARG, "mpm_cell_order_noalloc: np = " + std::to_string(d->np) +
                                      " exceeds MPM_NOALLOC_MAX_PARTICLES (" + std::to_string(NA_NP) + ")");
    if (d->nnx < 4 || d->nny < 4 || (d->dim == 3 && d->nnz < 4) || !(d->dx > 0) || !(d->dy > 0) ||
        (d->dim == 3 && !(d->dz > 0)))
        return na_fail(MPM_E_ARG, "mpm_cell_order_noalloc: invalid grid");
    int dev = 0;
    NA_CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= MAX_DEV) return na_fail(MPM_E_ARG, "mpm_cell_order_noalloc: device ordinal out of range");
    // set-up per device, with that device current: the scratch's device
    // address.  A failed lookup is not remembered, so a later call retries it.
    unsigned char *scratch = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_setup_mu);
        if (!g_scratch_ptr[dev]) {
            void *p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p)
                return na_fail(MPM_E_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
            g_scratch_ptr[dev] = (unsigned char *)p;
        }
        scratch = g_scratch_ptr[dev];
    }
    cudaStream_t st = (cudaStream_t)stream;
    return d->dim == 2 ? run<2>(d, x, y, z, order_out, p2c_out, st, scratch)
                       : run<3>(d, x, y, z, order_out, p2c_out, st, scratch);
}
