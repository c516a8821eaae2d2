// mpm_sort.cuh -- cell sort of the particles (no counterpart in the reference,
// which never reorders particles).
//
// Key: the particle's cell (the reference's p2c cell, Julia fld/cld rule)
// renumbered tile-major: tiles of tx x ty x tz cells (a run-time shape, 32
// cells by default so that one warp lane stands for one cell), key = tile *
// cpt + cell-in-tile.  Order: ascending tile; inside a tile ascending rank of
// the particle within its cell, then ascending cell-in-tile -- a CPU stable
// sort by (tile, rank, cell-in-tile).  The rank orders a cell's particles by
// their sub-cell octant (which half of the cell they sit in along each axis:
// bit 0 x, bit 1 y, bit 2 z), then by original index; on a regular lattice
// with two particles per cell and axis, rank r then holds the particles of
// one octant in every cell, whose uGIMP windows have the same shape.
//
// Counting sort: count per key, exclusive scan, scatter (atomic slot within
// the bucket), then each bucket is ordered by (octant, original index) (buckets
// hold the few particles of one cell), then every particle array is gathered
// through the permutation.
#pragma once
#include "mpm_kernels.cuh"

namespace mpm {

// default tile shapes (cells): one warp lane per cell
template <int D> struct Tile {
    static constexpr int TX = D == 3 ? 2 : 4, TY = 8, TZ = D == 3 ? 2 : 1;
    static constexpr int CPT = TX * TY * TZ;
};

struct SortGeom {
    int ncx, ncy, ncz;      // cells per axis
    int ntx, nty, ntz;      // tiles per axis
    int tx, ty, tz, cpt;    // tile shape (cells) and cells per tile
    uint32_t nk;            // number of keys = tiles * cpt
};

inline int64_t sort_cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }

// sort geometry of a grid of nnx x nny (x nnz) nodes in tiles of tx x ty (x tz)
// cells; returns the number of keys (tiles x cells per tile)
inline int64_t sort_geom(SortGeom &sg, int dim, int64_t nnx, int64_t nny, int64_t nnz, int tx, int ty, int tz) {
    sg.ncx = (int)(nnx - 1);
    sg.ncy = (int)(nny - 1);
    sg.ncz = dim == 3 ? (int)(nnz - 1) : 1;
    sg.tx = tx;
    sg.ty = ty;
    sg.tz = dim == 3 ? tz : 1;
    sg.cpt = sg.tx * sg.ty * sg.tz;
    sg.ntx = (int)sort_cdiv(sg.ncx, sg.tx);
    sg.nty = (int)sort_cdiv(sg.ncy, sg.ty);
    sg.ntz = dim == 3 ? (int)sort_cdiv(sg.ncz, sg.tz) : 1;
    const int64_t nk = (int64_t)sg.ntx * sg.nty * sg.ntz * sg.cpt;
    sg.nk = (uint32_t)nk;
    return nk;
}

// sort keys and original indices carry the octant in their top bits
constexpr int OCT_SHIFT = 29;
constexpr uint32_t LOW29 = (1u << OCT_SHIFT) - 1u;

template <int D> __device__ __forceinline__ uint32_t cell_key(int cx, int cy, int cz, const SortGeom &s) {
    int tx = cx / s.tx, ty = cy / s.ty, tz = D == 3 ? cz / s.tz : 0;
    int lx = cx - tx * s.tx, ly = cy - ty * s.ty, lz = D == 3 ? cz - tz * s.tz : 0;
    uint32_t t = (uint32_t)((tz * s.ntx + tx) * s.nty + ty);
    return t * (uint32_t)s.cpt + (uint32_t)((lz * s.tx + lx) * s.ty + ly);
}

// sub-cell octant of a particle in cell (cx, cy, cz): bit a set when its offset
// from the cell's first node is at least half a cell along axis a
template <int D, typename R>
__device__ __forceinline__ uint32_t cell_octant(const double *x, int cx, int cy, int cz, const GDev<R> &g) {
    uint32_t o = 0;
    if (cell_offset<R>(x[0], cx, g.ax[0]) >= 0.5 * g.ax[0].h) o |= 1u;
    if (cell_offset<R>(x[1], cy, g.ax[1]) >= 0.5 * g.ax[1].h) o |= 2u;
    if (D == 3 && cell_offset<R>(x[2], cz, g.ax[2]) >= 0.5 * g.ax[2].h) o |= 4u;
    return o;
}

template <int D, typename R>
__global__ void k_sort_keys(PDev<D, R> P, GDev<R> g, SortGeom sg, int64_t np, uint32_t *keys,
                            uint32_t *cnt) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    double x[3];
    load_x<D, R>(P, i, x);
    int ci[3];
    particle_cell<D, R>(x, g, ci);
    int cx = clampi(ci[0], 0, sg.ncx - 1), cy = clampi(ci[1], 0, sg.ncy - 1);
    int cz = D == 3 ? clampi(ci[2], 0, sg.ncz - 1) : 0;
    uint32_t k = cell_key<D>(cx, cy, cz, sg);
    keys[i] = k | (cell_octant<D, R>(x, cx, cy, cz, g) << OCT_SHIFT);
    atomicAdd(&cnt[k], 1u);
}

// ---- exclusive scan of uint32 counts (chunked reduce / top scan / down-sweep) ----
constexpr int SCAN_T = 256, SCAN_IT = 8, SCAN_CHUNK = SCAN_T * SCAN_IT;

__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t *tot) {
    __shared__ uint32_t ws[SCAN_T / 32];
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) ws[wid] = x;
    __syncthreads();
    if (wid == 0) {
        uint32_t s = lane < SCAN_T / 32 ? ws[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < SCAN_T / 32) ws[lane] = s;
    }
    __syncthreads();
    uint32_t base = wid > 0 ? ws[wid - 1] : 0;
    if (tot) *tot = ws[SCAN_T / 32 - 1];
    __syncthreads();
    return base + x - v;
}

static __global__ void __launch_bounds__(SCAN_T) k_scan_reduce(const uint32_t *in, uint32_t n, uint32_t *bsum) {
    uint32_t base = blockIdx.x * SCAN_CHUNK;
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_IT; ++k) {
        uint32_t i = base + k * SCAN_T + threadIdx.x;
        if (i < n) s += in[i];
    }
    uint32_t tot;
    block_excl_scan(s, &tot);
    if (threadIdx.x == 0) bsum[blockIdx.x] = tot;
}

static __global__ void __launch_bounds__(SCAN_T) k_scan_top(uint32_t *bsum, uint32_t nb) {
    uint32_t carry = 0;
    for (uint32_t base = 0; base < nb; base += SCAN_T) {
        uint32_t i = base + threadIdx.x;
        uint32_t v = i < nb ? bsum[i] : 0;
        uint32_t tot;
        uint32_t e = block_excl_scan(v, &tot);
        if (i < nb) bsum[i] = carry + e;
        carry += tot;
    }
}

// off[i] = exclusive prefix of in; off[n] = total
static __global__ void __launch_bounds__(SCAN_T) k_scan_down(const uint32_t *in, uint32_t n, const uint32_t *bsum,
                                                      uint32_t *off) {
    uint32_t base = blockIdx.x * SCAN_CHUNK + threadIdx.x * SCAN_IT;
    uint32_t v[SCAN_IT];
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_IT; ++k) {
        uint32_t i = base + k;
        v[k] = i < n ? in[i] : 0;
        s += v[k];
    }
    uint32_t tot;
    uint32_t e = block_excl_scan(s, &tot) + bsum[blockIdx.x];
#pragma unroll
    for (int k = 0; k < SCAN_IT; ++k) {
        uint32_t i = base + k;
        if (i < n) off[i] = e;
        e += v[k];
        if (i + 1 == n) off[n] = e;
    }
}

// scatter (orig index, old position) pairs into their buckets
template <int D, typename R>
__global__ void k_sort_scatter(PDev<D, R> P, int64_t np, const uint32_t *keys, const uint32_t *off,
                               uint32_t *cur, uint2 *pairs) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    const uint32_t kk = keys[i], k = kk & LOW29;
    uint32_t pos = off[k] + atomicAdd(&cur[k], 1u);
    pairs[pos] = make_uint2(P.orig[i] | (kk & ~LOW29), (uint32_t)i);
}

// order each bucket by (octant, original index) (the pair's first word);
// buckets above SMALL are queued for the CTA sort
constexpr int BUCKET_SMALL = 32;
constexpr int BUCKET_MAX = 4096;

static __global__ void k_sort_buckets(const uint32_t *off, uint32_t nk, uint2 *pairs, uint32_t *big,
                               uint32_t *nbig, uint32_t big_cap, int *err) {
    uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nk) return;
    uint32_t b = off[k], e = off[k + 1];
    uint32_t n = e - b;
    if (n < 2) return;
    if (n > BUCKET_SMALL) {
        if (n > BUCKET_MAX) { atomicOr(err, ERR_OVF); return; }
        uint32_t slot = atomicAdd(nbig, 1u);
        if (slot < big_cap) big[slot] = k;
        else atomicOr(err, ERR_OVF);
        return;
    }
    for (uint32_t a = b + 1; a < e; ++a) {
        uint2 t = pairs[a];
        uint32_t j = a;
        while (j > b && pairs[j - 1].x > t.x) { pairs[j] = pairs[j - 1]; --j; }
        pairs[j] = t;
    }
}

// bitonic sort of one large bucket in shared memory (one CTA per bucket)
static __global__ void __launch_bounds__(512) k_sort_big(const uint32_t *off, const uint32_t *big, const uint32_t *nbig,
                                                  uint32_t big_cap, uint2 *pairs) {
    __shared__ unsigned long long s[BUCKET_MAX];
    uint32_t nb = *nbig;
    if (nb > big_cap) nb = big_cap;
    for (uint32_t q = blockIdx.x; q < nb; q += gridDim.x) {
        uint32_t k = big[q];
        uint32_t b = off[k], n = off[k + 1] - b;
        uint32_t P2 = 1;
        while (P2 < n) P2 <<= 1;
        for (uint32_t i = threadIdx.x; i < P2; i += blockDim.x)
            s[i] = i < n ? ((unsigned long long)pairs[b + i].x << 32) | pairs[b + i].y : ~0ull;
        __syncthreads();
        for (uint32_t size = 2; size <= P2; size <<= 1)
            for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
                for (uint32_t i = threadIdx.x; i < P2; i += blockDim.x) {
                    uint32_t j = i ^ stride;
                    if (j > i) {
                        bool up = (i & size) == 0;
                        unsigned long long a = s[i], c = s[j];
                        if ((a > c) == up) { s[i] = c; s[j] = a; }
                    }
                }
                __syncthreads();
            }
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x)
            pairs[b + i] = make_uint2((uint32_t)(s[i] >> 32), (uint32_t)(s[i] & 0xffffffffu));
        __syncthreads();
    }
}

// list of the tiles that hold particles after a sort
static __global__ void k_tile_list(const uint32_t *off, uint32_t ntile, uint32_t cpt, uint32_t *tiles, uint32_t *ntiles) {
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntile) return;
    if (off[(t + 1) * cpt] > off[t * cpt]) tiles[atomicAdd(ntiles, 1u)] = t;
}

// Rank-major order inside each tile: the particles of a tile, ordered by
// (cell, original index) after the bucket sort, are regrouped as (rank within
// the cell, cell): the first particle of every cell, then the second one of
// every cell, ...  Adjacent threads then work on adjacent cells, so their
// stencils hit different nodes at the same time (no same-address conflicts in
// the shared-memory scatter) while loads stay coalesced.  One CTA of CPT
// threads (one per cell) per tile.
template <int CPT>
__global__ void __launch_bounds__(CPT) k_tile_transpose(const uint32_t *off, const uint32_t *tiles,
                                                        const uint32_t *ntiles, const uint2 *src, uint2 *dst) {
    __shared__ uint32_t ws[CPT / 32 + 1];
    __shared__ uint32_t s_max;
    const uint32_t nt = *ntiles;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (uint32_t q = blockIdx.x; q < nt; q += gridDim.x) {
        const uint32_t t = tiles[q];
        const uint32_t k = t * CPT + threadIdx.x;
        const uint32_t b = off[k], n = off[k + 1] - b;
        const uint32_t tile_base = off[t * CPT];
        if (threadIdx.x == 0) s_max = 0;
        __syncthreads();
        atomicMax(&s_max, n);
        __syncthreads();
        const uint32_t maxn = s_max;
        uint32_t level = tile_base;
        for (uint32_t r = 0; r < maxn; ++r) {
            uint32_t f = n > r ? 1u : 0u;
            uint32_t bal = __ballot_sync(0xffffffffu, f);
            uint32_t pre = __popc(bal & ((1u << lane) - 1u));
            if (lane == 0) ws[wid] = __popc(bal);
            __syncthreads();
            uint32_t before = 0, tot = 0;
            for (int w = 0; w < CPT / 32; ++w) {
                uint32_t c = ws[w];
                if (w < wid) before += c;
                tot += c;
            }
            if (f) dst[level + before + pre] = src[b + r];
            level += tot;
            __syncthreads();
        }
    }
}

// gather every particle array through the permutation (new k <- old pairs[k].y)
template <int D, typename R>
__global__ void k_permute(PDev<D, R> src, PDev<D, R> dst, const uint2 *pairs, int64_t np) {
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= np) return;
    uint2 pr = pairs[k];
    uint32_t o = pr.y;
    constexpr int NV = PDev<D, R>::NV, NF = PDev<D, R>::NF;
#pragma unroll
    for (int d = 0; d < D; ++d) { dst.x[d][k] = src.x[d][o]; dst.v[d][k] = src.v[d][o]; }
#pragma unroll
    for (int c = 0; c < NV; ++c) { dst.sig[c][k] = src.sig[c][o]; dst.eps[c][k] = src.eps[c][o]; }
#pragma unroll
    for (int c = 0; c < NF; ++c) dst.F[c][k] = src.F[c][o];
    dst.epsq[k] = src.epsq[o]; dst.epsk[k] = src.epsk[o]; dst.epsv[k] = src.epsv[o];
    dst.m[k] = src.m[o]; dst.vol0[k] = src.vol0[o]; dst.vol[k] = src.vol[o];
    dst.mat[k] = src.mat[o];
    if (src.coh) dst.coh[k] = src.coh[o];
    if (src.n) {
        dst.n[k] = src.n[o]; dst.sigw[k] = src.sigw[o]; dst.mw[k] = src.mw[o];
#pragma unroll
        for (int d = 0; d < D; ++d) dst.vw[d][k] = src.vw[d][o];
#pragma unroll
        for (int c = 0; c < NV; ++c) dst.epsw[c][k] = src.epsw[c][o];
    }
    dst.orig[k] = pr.x & LOW29;
}

}  // namespace mpm
