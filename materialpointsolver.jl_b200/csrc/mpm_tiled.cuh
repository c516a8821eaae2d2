// mpm_tiled.cuh -- shared-memory tiled particle passes.
//
// After a cell sort the particles of one tile of TX x TY x TZ cells are
// contiguous.  One CTA processes a tile at a time (persistent loop over the
// list of non-empty tiles):
//   * the node window the tile's particles can read -- cells widened by a
//     margin of MARGIN cells for the drift since the last sort, plus the
//     uGIMP stencil (-1 .. +2 nodes) -- is staged in shared memory with one
//     coalesced load per node, instead of one global gather per
//     particle-node pair (each node is read by ~27 particles);
//   * gathers (ΣN·vsT, ΣN·as, ΣΔu⊗∇N) then read shared memory;
//   * scatters (P2G mass / momentum / force, DM2 momentum) go straight to the
//     global node records with vector reductions: shared-memory float
//     atomics are slower than L2 reductions on this part;
//   * a particle whose stencil left the window (moved more than MARGIN cells
//     since the sort) gathers from global memory.
// The per-particle arithmetic is the one of mpm_kernels.cuh.
#pragma once
#include "mpm_sort.cuh"

namespace mpm {

constexpr int MARGIN = 1;

template <int D> struct Win {
    using T = Tile<D>;
    static constexpr int WX = T::TX + 2 * MARGIN + 3;
    static constexpr int WY = T::TY + 2 * MARGIN + 3;
    static constexpr int WZ = D == 3 ? T::TZ + 2 * MARGIN + 3 : 1;
    static constexpr int WN = WX * WY * WZ;
};

struct TileList {
    const uint32_t *tiles;   // ids of non-empty tiles
    const uint32_t *ntiles;  // their count (device)
    const uint32_t *off;     // particle offsets per sort key
    SortGeom sg;
};


template <int D> struct TileGeo {
    int c0[3];   // first cell of the tile
    int w0[3];   // first node of the window
};

// (the window is sized for the default tile shape; with a larger run-time
// shape the particles beyond it take the global path)
template <int D> __device__ __forceinline__ TileGeo<D> tile_geo(uint32_t t, const SortGeom &sg) {
    TileGeo<D> g;
    int ty = (int)(t % (uint32_t)sg.nty);
    uint32_t r = t / (uint32_t)sg.nty;
    int tx = (int)(r % (uint32_t)sg.ntx);
    int tz = (int)(r / (uint32_t)sg.ntx);
    g.c0[0] = tx * sg.tx; g.c0[1] = ty * sg.ty; g.c0[2] = D == 3 ? tz * sg.tz : 0;
    for (int a = 0; a < 3; ++a) g.w0[a] = g.c0[a] - MARGIN - 1;
    if (D == 2) g.w0[2] = 0;
    return g;
}

// window-local index of window node (lx, ly, lz); y fastest like the grid
template <int D> __device__ __forceinline__ int wl(int lx, int ly, int lz) {
    using W = Win<D>;
    return (lz * W::WX + lx) * W::WY + ly;
}

// is the particle's 3^D stencil inside the window?  returns local base
template <int D, typename R>
__device__ __forceinline__ bool in_window(const AxisW<R> *w, const TileGeo<D> &tg, int *lb) {
    using W = Win<D>;
    const int wn[3] = {W::WX, W::WY, W::WZ};
    bool ok = true;
#pragma unroll
    for (int a = 0; a < D; ++a) {
        lb[a] = w[a].base - tg.w0[a];
        ok = ok && lb[a] >= 0 && lb[a] + 2 < wn[a];
    }
    if (D == 2) lb[2] = 0;
    return ok;
}

template <int D, typename R>
__device__ __forceinline__ void mark_window(const GDev<R> &g, const TileGeo<D> &tg) {
    using B = Blk<D>;
    using W = Win<D>;
    int x0 = clampi(tg.w0[0], 0, g.nnx - 1) / B::BX, x1 = clampi(tg.w0[0] + W::WX - 1, 0, g.nnx - 1) / B::BX;
    int y0 = clampi(tg.w0[1], 0, g.nny - 1) / B::BY, y1 = clampi(tg.w0[1] + W::WY - 1, 0, g.nny - 1) / B::BY;
    int z0 = 0, z1 = 0;
    if (D == 3) { z0 = clampi(tg.w0[2], 0, g.nnz - 1) / B::BZ; z1 = clampi(tg.w0[2] + W::WZ - 1, 0, g.nnz - 1) / B::BZ; }
    int nx = x1 - x0 + 1, ny = y1 - y0 + 1, nz = z1 - z0 + 1;
    for (int k = threadIdx.x; k < nx * ny * nz; k += blockDim.x) {
        int by = y0 + k % ny, r = k / ny, bx = x0 + r % nx, bz = z0 + r / nx;
        mark_block<R>(g, (bz * g.nbx + bx) * g.nby + by);
    }
}

// global node of window node n (or -1 outside the grid)
template <int D, typename R>
__device__ __forceinline__ int window_global(const GDev<R> &g, const TileGeo<D> &tg, int n) {
    using W = Win<D>;
    int ly = n % W::WY, r = n / W::WY, lx = r % W::WX, lz = r / W::WX;
    int ix = tg.w0[0] + lx, iy = tg.w0[1] + ly, iz = tg.w0[2] + lz;
    if (ix < 0 || ix >= g.nnx || iy < 0 || iy >= g.nny) return -1;
    if (D == 3 && (iz < 0 || iz >= g.nnz)) return -1;
    return node_id<D>(ix, iy, iz, g.nnx, g.nny);
}



// G2P gathers of one particle from the window in shared memory (SMEM) or from
// the global node records: tT = ΣN·vsT, dF = Σ(Δu - Δu_c)⊗∇N (Σ∇N = 0).
template <int D, typename R, bool SMEM>
__device__ __forceinline__ void g2p_gather(const GDev<R> &g, const AxisW<R> *w, const int *lb, int n0,
                                           const R *s_vT, const R *s_du, R *tT, R *dF) {
    using W = Win<D>;
    constexpr int NC = D == 3 ? 3 : 1;
    const int plane = g.nnx * g.nny;
    R ucx, ucy, ucz;
    if (SMEM) {
        int n = wl<D>(lb[0] + 1, lb[1] + 1, lb[2] + (D == 3 ? 1 : 0));
        ucx = s_du[n]; ucy = s_du[W::WN + n]; ucz = s_du[2 * W::WN + n];
    } else {
        const auto qc = g.gat[n0 + g.nny + 1 + (D == 3 ? plane : 0)].b;
        ucx = qc.x; ucy = qc.y; ucz = qc.z;
    }
#pragma unroll
    for (int c = 0; c < NC; ++c)
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                R Nz = D == 3 ? w[2].N[c] : R(1);
                R N = D == 3 ? w[0].N[a] * w[1].N[b] * Nz : w[0].N[a] * w[1].N[b];
                R vx, vy, vz, ux, uy, uz;
                if (SMEM) {
                    int n = wl<D>(lb[0] + a, lb[1] + b, lb[2] + c);
                    vx = s_vT[n]; vy = s_vT[W::WN + n]; vz = s_vT[2 * W::WN + n];
                    ux = s_du[n]; uy = s_du[W::WN + n]; uz = s_du[2 * W::WN + n];
                } else {
                    const Node8<R> r = g.gat[n0 + a * g.nny + b + c * plane];
                    vx = r.a.x; vy = r.a.y; vz = r.a.z; ux = r.b.x; uy = r.b.y; uz = r.b.z;
                }
                ux -= ucx; uy -= ucy; uz -= ucz;
                tT[0] += N * vx; tT[1] += N * vy;
                if (D == 3) tT[2] += N * vz;
                if (D == 2) {
                    R gx = w[0].dN[a] * w[1].N[b];
                    R gy = w[1].dN[b] * w[0].N[a];
                    dF[0] += ux * gx; dF[1] += ux * gy;
                    dF[2] += uy * gx; dF[3] += uy * gy;
                } else {
                    R gx = w[0].dN[a] * w[1].N[b] * Nz;
                    R gy = w[1].dN[b] * w[0].N[a] * Nz;
                    R gz = w[2].dN[c] * w[0].N[a] * w[1].N[b];
                    dF[0] += ux * gx; dF[1] += ux * gy; dF[2] += ux * gz;
                    dF[3] += uy * gx; dF[4] += uy * gy; dF[5] += uy * gz;
                    dF[6] += uz * gx; dF[7] += uz * gy; dF[8] += uz * gz;
                }
            }
}

// DM1 gathers of one particle: tT = ΣN·vsT, ta = ΣN·as, tv = ΣN·vs.
template <int D, typename R, bool SMEM>
__device__ __forceinline__ void dm_gather(const GDev<R> &g, const StepParams &sp, const AxisW<R> *w, const int *lb,
                                          int n0, const R *s_vT, const R *s_as, const R *s_vs, R *tT, R *ta, R *tv) {
    using W = Win<D>;
    using T4 = typename Vec<R>::T4;
    constexpr int NC = D == 3 ? 3 : 1;
    const int plane = g.nnx * g.nny;
#pragma unroll
    for (int c = 0; c < NC; ++c)
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                R N = D == 3 ? w[0].N[a] * w[1].N[b] * w[2].N[c] : w[0].N[a] * w[1].N[b];
                R vx, vy, vz, ax, ay, az, sx = 0, sy = 0, sz = 0;
                if (SMEM) {
                    int n = wl<D>(lb[0] + a, lb[1] + b, lb[2] + c);
                    vx = s_vT[n]; vy = s_vT[W::WN + n]; vz = s_vT[2 * W::WN + n];
                    ax = s_as[n]; ay = s_as[W::WN + n]; az = s_as[2 * W::WN + n];
                    if (sp.need_vs) { sx = s_vs[n]; sy = s_vs[W::WN + n]; sz = s_vs[2 * W::WN + n]; }
                } else {
                    int n = n0 + a * g.nny + b + c * plane;
                    const Node8<R> r = g.gat[n];
                    vx = r.a.x; vy = r.a.y; vz = r.a.z; ax = r.b.x; ay = r.b.y; az = r.b.z;
                    if (sp.need_vs) { T4 q3 = g.gvs[n]; sx = q3.x; sy = q3.y; sz = q3.z; }
                }
                tT[0] += N * vx; tT[1] += N * vy; tT[2] += N * vz;
                ta[0] += N * ax; ta[1] += N * ay; ta[2] += N * az;
                tv[0] += N * sx; tv[1] += N * sy; tv[2] += N * sz;
            }
}

// ---------------------------------------------------------------------------
// Tiled double mapping (DM1 velocity + DM2 momentum re-scatter).
// smem: vsT, as (+ vs) of the window, structure of arrays.
// ---------------------------------------------------------------------------
template <int D, typename R>
__global__ void __launch_bounds__(256, MPM_P_MINB) k_dmap_tile(PDev<D, R> P, GDev<R> g, StepParams sp, TileList tl) {
    using W = Win<D>;
    using T4 = typename Vec<R>::T4;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R *s_vT = (R *)smem_raw;                 // 3 x WN
    R *s_as = s_vT + 3 * W::WN;              // 3 x WN
    R *s_vs = s_as + 3 * W::WN;              // 3 x WN (only if need_vs)
    const uint32_t nt = *tl.ntiles;
    constexpr int NC = D == 3 ? 3 : 1;
    const int plane = g.nnx * g.nny;
    for (uint32_t q = blockIdx.x; q < nt; q += gridDim.x) {
        const uint32_t t = tl.tiles[q];
        const TileGeo<D> tg = tile_geo<D>(t, tl.sg);
        const uint32_t p0 = tl.off[t * (uint32_t)tl.sg.cpt], p1 = tl.off[(t + 1) * (uint32_t)tl.sg.cpt];
        for (int n = threadIdx.x; n < W::WN; n += blockDim.x) {
            int gn = window_global<D, R>(g, tg, n);
            Node8<R> r;
            if (gn >= 0) r = g.gat[gn];
            else { r.a = mk4<R>(0, 0, 0, 0); r.b = r.a; }
            s_vT[n] = r.a.x; s_vT[W::WN + n] = r.a.y; s_vT[2 * W::WN + n] = r.a.z;
            s_as[n] = r.b.x; s_as[W::WN + n] = r.b.y; s_as[2 * W::WN + n] = r.b.z;
            if (sp.need_vs) {
                T4 vs = gn >= 0 ? g.gvs[gn] : mk4<R>(0, 0, 0, 0);
                s_vs[n] = vs.x; s_vs[W::WN + n] = vs.y; s_vs[2 * W::WN + n] = vs.z;
            }
        }
        __syncthreads();
        for (uint32_t i = p0 + threadIdx.x; i < p1; i += blockDim.x) {
            double x[3];
            load_x<D, R>(P, i, x);
            R vo[3];
#pragma unroll
            for (int d = 0; d < D; ++d) vo[d] = ldcs(P.v[d] + i);
            const R m = ldcs(P.m + i);
            AxisW<R> w[3];
            particle_weights<D, R>(x, g, w);
            int lb[3];
            const bool inw = in_window<D, R>(w, tg, lb);
            const int n0 = window_n0<D, R>(g, w);
            R tT[3] = {0, 0, 0}, ta[3] = {0, 0, 0}, tv[3] = {0, 0, 0};
            if (inw) dm_gather<D, R, true>(g, sp, w, lb, n0, s_vT, s_as, s_vs, tT, ta, tv);
            else dm_gather<D, R, false>(g, sp, w, lb, n0, s_vT, s_as, s_vs, tT, ta, tv);
            const R dt = (R)sp.dt, FLIP = (R)sp.FLIP, PIC = (R)sp.PIC;
            R vn[3] = {0, 0, 0};
#pragma unroll
            for (int d = 0; d < D; ++d) {
                if (sp.va == 0) vn[d] = FLIP * vo[d] + PIC * tv[d] + ta[d] * dt;
                else vn[d] = FLIP * (vo[d] + (tT[d] - tv[d])) + PIC * tT[d];
                stcs(P.v[d] + i, vn[d]);
            }
            const R p[3] = {m * vn[0], m * vn[1], D == 3 ? m * vn[2] : R(0)};
#pragma unroll
            for (int c = 0; c < NC; ++c)
#pragma unroll
                for (int a = 0; a < 3; ++a)
#pragma unroll
                    for (int b = 0; b < 3; ++b) {
                        R N = D == 3 ? w[0].N[a] * w[1].N[b] * w[2].N[c] : w[0].N[a] * w[1].N[b];
                        const int n = n0 + a * g.nny + b + c * plane;
                        if (N != R(0)) red_add4(&g.acc[n].a, R(0), p[0] * N, p[1] * N, p[2] * N);
                    }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Tiled G2P + stress + position update, fused with the next step's P2G.
// smem: vsT and Δu of the window, structure of arrays.
// ---------------------------------------------------------------------------
template <int D, typename R, bool MC3 = false>
__global__ void __launch_bounds__(256, MPM_P_MINB) k_g2p_tile(PDev<D, R> P, GDev<R> g, StepParams sp, TileList tl) {
    using W = Win<D>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R *s_vT = (R *)smem_raw;          // 3 x WN
    R *s_du = s_vT + 3 * W::WN;       // 3 x WN
    const uint32_t nt = *tl.ntiles;
    const int plane = g.nnx * g.nny;
    for (uint32_t q = blockIdx.x; q < nt; q += gridDim.x) {
        const uint32_t t = tl.tiles[q];
        const TileGeo<D> tg = tile_geo<D>(t, tl.sg);
        const uint32_t p0 = tl.off[t * (uint32_t)tl.sg.cpt], p1 = tl.off[(t + 1) * (uint32_t)tl.sg.cpt];
        for (int n = threadIdx.x; n < W::WN; n += blockDim.x) {
            int gn = window_global<D, R>(g, tg, n);
            Node8<R> r;
            if (gn >= 0) r = g.gat[gn];
            else { r.a = mk4<R>(0, 0, 0, 0); r.b = r.a; }
            s_vT[n] = r.a.x; s_vT[W::WN + n] = r.a.y; s_vT[2 * W::WN + n] = r.a.z;
            s_du[n] = r.b.x; s_du[W::WN + n] = r.b.y; s_du[2 * W::WN + n] = r.b.z;
        }
        __syncthreads();
        for (uint32_t i = p0 + threadIdx.x; i < p1; i += blockDim.x) {
            double x[3];
            load_x<D, R>(P, i, x);
            AxisW<R> w[3];
            particle_weights<D, R>(x, g, w);
            int lb[3];
            const bool inw = in_window<D, R>(w, tg, lb);
            const int n0 = window_n0<D, R>(g, w);
            R tT[3] = {0, 0, 0};
            R dF[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            if (inw) g2p_gather<D, R, true>(g, w, lb, n0, s_vT, s_du, tT, dF);
            else g2p_gather<D, R, false>(g, w, lb, n0, s_vT, s_du, tT, dF);
            R s[6], vol;
            update_particle<D, R, MC3>(P, g, sp, i, x, tT, dF, s, vol);
            // next step's P2G at the new position, straight into the node records
            if (!particle_weights<D, R>(x, g, w)) { atomicOr(g.err, ERR_OOG); continue; }
            R v[3];
#pragma unroll
            for (int d = 0; d < D; ++d) v[d] = ldcs(P.v[d] + i);
            if (D == 2) v[2] = R(0);
            p2g_scatter<D, R>(g, w, ldcs(P.m + i), vol, v, s, (R)sp.G);
        }
        __syncthreads();
    }
}

}  // namespace mpm
