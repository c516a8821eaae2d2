// mpm_box.cuh -- the FP32 particle passes with the node data of a tile in
// shared memory: one warp per tile, one lane per cell.
//
// After the cell sort the particles of a tile of 32 cells are contiguous and
// rank-major: rank 0 (the first particle, by sub-cell octant then original
// index) of every non-empty cell, then rank 1, ...  One warp takes a whole
// tile (a persistent loop over the list of non-empty tiles, fetched by an
// atomic counter) and walks its ranks; in rank r lane l holds the r-th
// particle of cell l, so the lanes of a warp are 32 distinct cells.
//
// Each warp owns two boxes of the tile's nodes in shared memory, the
// (tx + 3) x (ty + 3) x (tz + 3) nodes a particle of the tile can reach (its
// uGIMP window starts at most one node below its cell):
//   * the gather box, filled once per tile from the node records (the G2P
//     pass reads Δus and vsT, the double mapping as); every particle-node
//     read of the pass is then a shared-memory load;
//   * the scatter box, which accumulates the tile's P2G (mass, momentum,
//     force) or DM2 (momentum) contributions with plain read-modify-writes
//     and is added to the node records once, with one vector reduction per
//     node and record, when the tile is done -- instead of one reduction per
//     particle-node pair.  (Shared-memory FP32 atomics are compare-and-swap
//     loops on this part; plain read-modify-writes need no atomics because
//     one warp owns the box and no two of its lanes write one node at once.)
// Two lanes write the same node in the same instruction only if their
// windows start at the same node.  Lanes hold distinct cells and, after the
// sort, particles of one octant, whose windows start at distinct nodes; a
// particle that has since crossed a cell centre can meet another lane's
// window.  Such lanes are detected per rank (__match_any_sync on the window
// corner) and scatter in successive rounds.  Windows of neighbouring lanes do
// overlap (lane L's row 1 is lane L+1's row 0), so one node is updated by
// different lanes at different window offsets: every node update is followed
// by __syncwarp over the scattering lanes, which orders it before the next
// offset's loads of the other lanes (without it the compiler may hoist those
// loads above the stores).  A particle whose window reaches
// outside the box (it drifted more than half a cell out of its tile since the
// sort) gathers from and reduces into the global node records directly, like
// the per-particle kernels.
//
// The arithmetic per particle is the one of mpm_kernels.cuh (same functions),
// only the summation order of the nodal sums differs.
#pragma once
#include "mpm_sort.cuh"

// warps per CTA and resident CTAs per SM of the box passes
#ifndef MPM_BOX_WARPS
#define MPM_BOX_WARPS 4
#endif
#ifndef MPM_BOX_G2P_MINB
#define MPM_BOX_G2P_MINB 3
#endif
#ifndef MPM_BOX_DMAP_MINB
#define MPM_BOX_DMAP_MINB 6
#endif

namespace mpm {

// Box geometry of a tile of TX x TY x TZ cells (32 cells: one lane per cell).
template <int D, int TX_, int TY_, int TZ_> struct BoxGeo {
    static constexpr int TX = TX_, TY = TY_, TZ = D == 3 ? TZ_ : 1;
    static_assert(TX * TY * TZ == 32, "one lane per cell");
    static constexpr int BX = TX + 3, BY = TY + 3, BZ = D == 3 ? TZ + 3 : 1;
    static constexpr int BN = BX * BY * BZ;
    // fused pass: gather {Δu, vsT.x} + {vsT.y, vsT.z}; scatter {m, p} + {f, 0}
    static constexpr int G2_OFF = 16 * BN;
    static constexpr int SA_OFF = G2_OFF + ((8 * BN + 15) / 16) * 16;
    static constexpr int SB_OFF = SA_OFF + 16 * BN;
    static constexpr int G2P_BYTES = SB_OFF + 16 * BN;
    // double mapping: gather {as, 0}; scatter {p, 0}
    static constexpr int DM_BYTES = 32 * BN;
};

struct BoxTiles {
    const uint32_t *tiles;    // non-empty tiles
    const uint32_t *ntiles;   // their count (device)
    const uint32_t *off;      // particle offset per sort key (nk + 1)
    uint32_t *work;           // tile counter of this launch (zeroed before it)
    SortGeom sg;
};

// first cell of tile t (the key layout of cell_key)
template <int D> __device__ __forceinline__ void box_tile_origin(uint32_t t, const SortGeom &sg, int *c0) {
    const int ty = (int)(t % (uint32_t)sg.nty);
    const uint32_t r = t / (uint32_t)sg.nty;
    const int tx = (int)(r % (uint32_t)sg.ntx), tz = (int)(r / (uint32_t)sg.ntx);
    c0[0] = tx * sg.tx;
    c0[1] = ty * sg.ty;
    c0[2] = D == 3 ? tz * sg.tz : 0;
}

// next tile of this warp (all lanes get the same answer)
__device__ __forceinline__ uint32_t box_next_tile(const BoxTiles &bt) {
    uint32_t q = 0;
    if ((threadIdx.x & 31) == 0) q = atomicAdd(bt.work, 1u);
    return __shfl_sync(0xffffffffu, q, 0);
}

// global node of box node n (box origin b0), or -1 outside the grid
template <typename G, int D>
__device__ __forceinline__ int box_global(const GDev<float> &g, const int *b0, int n) {
    const int ly = n % G::BY, r = n / G::BY, lx = r % G::BX, lz = r / G::BX;
    const int ix = b0[0] + lx, iy = b0[1] + ly, iz = b0[2] + lz;
    if (ix < 0 || ix >= g.nnx || iy < 0 || iy >= g.nny) return -1;
    if (D == 3 && (iz < 0 || iz >= g.nnz)) return -1;
    return node_id<D>(ix, iy, iz, g.nnx, g.nny);
}

// window corner of a particle relative to the box; true if the window is inside
template <typename G, int D>
__device__ __forceinline__ bool box_window(const AxisW<float> *w, const int *b0, int *lb) {
    const int bn[3] = {G::BX, G::BY, G::BZ};
    bool in = true;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        lb[a] = a < D ? w[a].base - b0[a] : 0;
        if (a < D) in = in && lb[a] >= 0 && lb[a] + 2 < bn[a];
    }
    return in;
}

template <typename G> __device__ __forceinline__ int box_lin(int lx, int ly, int lz) {
    return (lz * G::BX + lx) * G::BY + ly;
}

// flag the node blocks the box overlaps (the node passes visit them)
template <typename G, int D> __device__ __forceinline__ void box_mark(const GDev<float> &g, const int *b0) {
    using B = Blk<D>;
    const int x0 = clampi(b0[0], 0, g.nnx - 1) / B::BX, x1 = clampi(b0[0] + G::BX - 1, 0, g.nnx - 1) / B::BX;
    const int y0 = clampi(b0[1], 0, g.nny - 1) / B::BY, y1 = clampi(b0[1] + G::BY - 1, 0, g.nny - 1) / B::BY;
    int z0 = 0, z1 = 0;
    if (D == 3) {
        z0 = clampi(b0[2], 0, g.nnz - 1) / B::BZ;
        z1 = clampi(b0[2] + G::BZ - 1, 0, g.nnz - 1) / B::BZ;
    }
    const int nx = x1 - x0 + 1, ny = y1 - y0 + 1, nz = z1 - z0 + 1;
    for (int k = threadIdx.x & 31; k < nx * ny * nz; k += 32) {
        const int by = y0 + k % ny, r = k / ny, bx = x0 + r % nx, bz = z0 + r / nx;
        mark_block<float>(g, (bz * g.nbx + bx) * g.nby + by);
    }
}

// ---- G2P gathers --------------------------------------------------------------------
// tT = ΣN·vsT, dF = Σ(Δu - Δu_c)⊗∇N (Σ∇N = 0; Δu_c: the window centre node), from
// the gather box (3D: g4 = {Δu, vsT.x}, g2 = {vsT.y, vsT.z}; 2D: g4 = {Δu, vsT}) ...
template <typename G, int D>
__device__ __forceinline__ void gather_box(const float4 *g4, const float2 *g2, const AxisW<float> *w, const int *lb,
                                           float *tT, float *dF) {
    constexpr int NC = D == 3 ? 3 : 1;
    const float4 cen = g4[box_lin<G>(lb[0] + 1, lb[1] + 1, D == 3 ? lb[2] + 1 : 0)];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        const float wz = D == 3 ? w[2].N[c] : 1.0f, gz = D == 3 ? w[2].dN[c] : 0.0f;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const float wx = w[0].N[a];
            const int col = box_lin<G>(lb[0] + a, lb[1], lb[2] + (D == 3 ? c : 0));
            float2 T01 = make_float2(0.f, 0.f), A01 = T01, B01 = T01;
            float T2 = 0.f, A2 = 0.f, B2 = 0.f;
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                const float wy = w[1].N[b], gy = w[1].dN[b];
                const float4 q = g4[col + b];
                const float2 w2 = make_float2(wy, wy), gg = make_float2(gy, gy);
                const float2 u01 = __fadd2_rn(make_float2(q.x, q.y), make_float2(-cen.x, -cen.y));
                A01 = __ffma2_rn(w2, u01, A01);
                B01 = __ffma2_rn(gg, u01, B01);
                if (D == 3) {
                    const float2 r = g2[col + b];
                    T01 = __ffma2_rn(w2, make_float2(q.w, r.x), T01);
                    T2 += wy * r.y;
                    const float u2 = q.z - cen.z;
                    A2 += wy * u2;
                    B2 += gy * u2;
                } else {
                    T01 = __ffma2_rn(w2, make_float2(q.z, q.w), T01);
                }
            }
            const float wxz = wx * wz, gxz = w[0].dN[a] * wz;
            tT[0] += wxz * T01.x;
            tT[1] += wxz * T01.y;
            if (D == 2) {
                dF[0] += gxz * A01.x; dF[1] += wxz * B01.x;
                dF[2] += gxz * A01.y; dF[3] += wxz * B01.y;
            } else {
                tT[2] += wxz * T2;
                const float xdz = wx * gz;
                const float A[3] = {A01.x, A01.y, A2}, Bv[3] = {B01.x, B01.y, B2};
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    dF[3 * k + 0] += gxz * A[k];
                    dF[3 * k + 1] += wxz * Bv[k];
                    dF[3 * k + 2] += xdz * A[k];
                }
            }
        }
    }
}

// ... or from the global node records (a window outside the box)
template <int D>
__device__ __forceinline__ void gather_global(const GDev<float> &g, const AxisW<float> *w, float *tT, float *dF) {
    constexpr int NC = D == 3 ? 3 : 1;
    const int n0 = window_n0<D, float>(g, w);
    const int plane = g.nnx * g.nny;
    const float4 cen = g.gat[n0 + g.nny + 1 + (D == 3 ? plane : 0)].b;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        const float wz = D == 3 ? w[2].N[c] : 1.0f, gz = D == 3 ? w[2].dN[c] : 0.0f;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const float wx = w[0].N[a];
            const int col = n0 + a * g.nny + (D == 3 ? c * plane : 0);
            float T[3] = {0, 0, 0}, A[3] = {0, 0, 0}, Bv[3] = {0, 0, 0};
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                const float wy = w[1].N[b], gy = w[1].dN[b];
                const Node8<float> q = g.gat[col + b];
                const float u[3] = {q.b.x - cen.x, q.b.y - cen.y, q.b.z - cen.z};
                T[0] += wy * q.a.x; T[1] += wy * q.a.y; T[2] += wy * q.a.z;
#pragma unroll
                for (int k = 0; k < D; ++k) { A[k] += wy * u[k]; Bv[k] += gy * u[k]; }
            }
            const float wxz = wx * wz, gxz = w[0].dN[a] * wz;
#pragma unroll
            for (int k = 0; k < D; ++k) tT[k] += wxz * T[k];
            if (D == 2) {
                dF[0] += gxz * A[0]; dF[1] += wxz * Bv[0];
                dF[2] += gxz * A[1]; dF[3] += wxz * Bv[1];
            } else {
                const float xdz = wx * gz;
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    dF[3 * k + 0] += gxz * A[k];
                    dF[3 * k + 1] += wxz * Bv[k];
                    dF[3 * k + 2] += xdz * A[k];
                }
            }
        }
    }
}

// ---- P2G into the scatter box (P2G_OS!, utils_OS.jl:424-496) --------------------------
// Node value = Ny·(m, p, X) + dNy·(0, 0, Y) per (x, z) window column, with
// σv = -Ω·σ: X_k = σv_kx·dNx·Nz + σv_kz·Nx·dNz (+ m·Nx·Nz·g on the last axis),
// Y_k = σv_ky·Nx·Nz (the separable form of p2g_scatter).
template <typename G, int D>
__device__ __forceinline__ void scatter_box(float4 *sa, float4 *sb, const AxisW<float> *w, const int *lb, float m,
                                            float vol, const float *v, const float *s, float grav,
                                            unsigned lanes) {
    constexpr int NC = D == 3 ? 3 : 1;
    const float p[3] = {m * v[0], m * v[1], D == 3 ? m * v[2] : 0.0f};
    float sv[6];
    if (D == 2) {
        sv[0] = -vol * s[0]; sv[1] = -vol * s[1]; sv[3] = -vol * s[3];
        sv[2] = sv[4] = sv[5] = 0.0f;
    } else {
#pragma unroll
        for (int k = 0; k < 6; ++k) sv[k] = -vol * s[k];
    }
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        const float wz = D == 3 ? w[2].N[c] : 1.0f, gz = D == 3 ? w[2].dN[c] : 0.0f;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const float wx = w[0].N[a];
            const float wxz = wx * wz, gxz = w[0].dN[a] * wz, xdz = wx * gz;
            float U[7], Y[3];
            U[0] = m * wxz;
            U[1] = p[0] * wxz; U[2] = p[1] * wxz; U[3] = p[2] * wxz;
            if (D == 2) {
                U[4] = sv[0] * gxz; U[5] = sv[3] * gxz + U[0] * grav; U[6] = 0.0f;
                Y[0] = sv[3] * wxz; Y[1] = sv[1] * wxz; Y[2] = 0.0f;
            } else {
                U[4] = sv[0] * gxz + sv[5] * xdz;
                U[5] = sv[3] * gxz + sv[4] * xdz;
                U[6] = sv[5] * gxz + sv[2] * xdz + U[0] * grav;
                Y[0] = sv[3] * wxz; Y[1] = sv[1] * wxz; Y[2] = sv[4] * wxz;
            }
            const float2 U01 = make_float2(U[0], U[1]), U23 = make_float2(U[2], U[3]);
            const float2 U45 = make_float2(U[4], U[5]), Y01 = make_float2(Y[0], Y[1]);
            const int col = box_lin<G>(lb[0] + a, lb[1], lb[2] + (D == 3 ? c : 0));
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                const float wy = w[1].N[b], gy = w[1].dN[b];
                const float2 w2 = make_float2(wy, wy), g2 = make_float2(gy, gy);
                const float4 A = sa[col + b];
                const float2 a01 = __ffma2_rn(w2, U01, make_float2(A.x, A.y));
                const float2 a23 = __ffma2_rn(w2, U23, make_float2(A.z, A.w));
                sa[col + b] = make_float4(a01.x, a01.y, a23.x, a23.y);
                const float4 B = sb[col + b];
                const float2 b01 = __ffma2_rn(g2, Y01, __ffma2_rn(w2, U45, make_float2(B.x, B.y)));
                const float b2 = fmaf(gy, Y[2], fmaf(wy, U[6], B.z));
                sb[col + b] = make_float4(b01.x, b01.y, b2, 0.0f);
                __syncwarp(lanes);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// G2P_OS! + DM1 position + liE!/dpP!/mcP! + the next step's P2G (the FUSE pass
// of k_g2p_chain), one warp per tile.
// ---------------------------------------------------------------------------
template <int D, int TX, int TY, int TZ, bool MC3>
__global__ void __launch_bounds__(MPM_BOX_WARPS * 32, MPM_BOX_G2P_MINB)
    k_g2p_box(PDev<D, float> P, GDev<float> g, StepParams sp, BoxTiles bt) {
    using G = BoxGeo<D, TX, TY, TZ>;
    extern __shared__ __align__(16) unsigned char box_smem[];
    const int lane = threadIdx.x & 31;
    const unsigned FULL = 0xffffffffu, lt = (1u << lane) - 1u;
    unsigned char *mine = box_smem + (threadIdx.x >> 5) * G::G2P_BYTES;
    float4 *g4 = reinterpret_cast<float4 *>(mine);
    float2 *g2 = reinterpret_cast<float2 *>(mine + G::G2_OFF);
    float4 *sa = reinterpret_cast<float4 *>(mine + G::SA_OFF);
    float4 *sb = reinterpret_cast<float4 *>(mine + G::SB_OFF);
    for (int n = lane; n < G::BN; n += 32) {
        sa[n] = make_float4(0.f, 0.f, 0.f, 0.f);
        sb[n] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    const uint32_t ntiles = *bt.ntiles;
    const float grav = (float)sp.G;
    for (uint32_t q = box_next_tile(bt); q < ntiles; q = box_next_tile(bt)) {
        const uint32_t t = bt.tiles[q];
        int b0[3];
        box_tile_origin<D>(t, bt.sg, b0);
        b0[0] -= 1; b0[1] -= 1;
        if (D == 3) b0[2] -= 1;
        // gather box: Δus (second half of the record, written by DM3) and vsT
        for (int n = lane; n < G::BN; n += 32) {
            const int gi = box_global<G, D>(g, b0, n);
            float4 a = make_float4(0.f, 0.f, 0.f, 0.f), b = a;
            if (gi >= 0) { const Node8<float> r = g.gat[gi]; a = r.a; b = r.b; }
            if (D == 3) {
                g4[n] = make_float4(b.x, b.y, b.z, a.x);
                g2[n] = make_float2(a.y, a.z);
            } else {
                g4[n] = make_float4(b.x, b.y, a.x, a.y);
            }
        }
        const uint32_t k0 = t * 32u;
        const uint32_t cnt = bt.off[k0 + lane + 1] - bt.off[k0 + lane];
        uint32_t row = bt.off[k0];
        const uint32_t maxc = __reduce_max_sync(FULL, cnt);
        __syncwarp();
        for (uint32_t r = 0; r < maxc; ++r) {
            const bool act = cnt > r;
            const unsigned bal = __ballot_sync(FULL, act);
            const int64_t i = (int64_t)row + __popc(bal & lt);
            row += __popc(bal);
            bool live = act;
            AxisW<float> w[3];
            int lb[3] = {0, 0, 0};
            bool inside = false;
            float s[6] = {0, 0, 0, 0, 0, 0}, vol = 0.f, v[3] = {0, 0, 0}, m = 0.f;
            if (act) {
                double x[3];
                load_x<D, float>(P, i, x);
                particle_weights<D, float>(x, g, w);   // out-of-grid particles get zero weights
                float tT[3] = {0, 0, 0}, dF[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
                if (box_window<G, D>(w, b0, lb)) gather_box<G, D>(g4, g2, w, lb, tT, dF);
                else gather_global<D>(g, w, tT, dF);
                update_particle<D, float, MC3>(P, g, sp, i, x, tT, dF, s, vol, nullptr);
                if (!particle_weights<D, float>(x, g, w)) {
                    atomicOr(g.err, ERR_OOG);
                    live = false;
                } else {
#pragma unroll
                    for (int d = 0; d < D; ++d) v[d] = ldcs(P.v[d] + i);
                    m = ldcs(P.m + i);
                    inside = box_window<G, D>(w, b0, lb);
                }
            }
            // lanes whose windows start at the same node scatter in successive rounds
            const int key = (live && inside) ? box_lin<G>(lb[0], lb[1], lb[2]) : -1 - lane;
            const unsigned same = __match_any_sync(FULL, key);
            const int grank = __popc(same & lt);
            const int rounds = __reduce_max_sync(FULL, (live && inside) ? grank : 0);
            for (int rr = 0; rr <= rounds; ++rr) {
                const bool mine = live && inside && grank == rr;
                const unsigned lanes = __ballot_sync(FULL, mine);
                if (mine) scatter_box<G, D>(sa, sb, w, lb, m, vol, v, s, grav, lanes);
                __syncwarp();
            }
            if (live && !inside) p2g_scatter<D, float>(g, w, m, vol, v, s, grav);
        }
        // the tile's nodal sums into the node records, one reduction per record
        __syncwarp();
        for (int n = lane; n < G::BN; n += 32) {
            const float4 a = sa[n], b = sb[n];
            if (a.x != 0.f || a.y != 0.f || a.z != 0.f || a.w != 0.f || b.x != 0.f || b.y != 0.f || b.z != 0.f) {
                const int gi = box_global<G, D>(g, b0, n);
                if (gi >= 0) {
                    red_add4(&g.acc[gi].a, a.x, a.y, a.z, a.w);
                    red_add4(&g.acc[gi].b, b.x, b.y, b.z, 0.f);
                }
                sa[n] = make_float4(0.f, 0.f, 0.f, 0.f);
                sb[n] = make_float4(0.f, 0.f, 0.f, 0.f);
            }
        }
        box_mark<G, D>(g, b0);
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// doublemapping1_a_OS! (velocity) + doublemapping2_OS! (momentum re-scatter),
// va = :a without the PIC term (FLIP only), one warp per tile.
// ---------------------------------------------------------------------------
template <int D, int TX, int TY, int TZ>
__global__ void __launch_bounds__(MPM_BOX_WARPS * 32, MPM_BOX_DMAP_MINB)
    k_dmap_box(PDev<D, float> P, GDev<float> g, StepParams sp, BoxTiles bt) {
    using G = BoxGeo<D, TX, TY, TZ>;
    constexpr int NC = D == 3 ? 3 : 1;
    extern __shared__ __align__(16) unsigned char box_smem[];
    const int lane = threadIdx.x & 31;
    const unsigned FULL = 0xffffffffu, lt = (1u << lane) - 1u;
    unsigned char *mine = box_smem + (threadIdx.x >> 5) * G::DM_BYTES;
    float4 *ga = reinterpret_cast<float4 *>(mine);
    float4 *sp4 = reinterpret_cast<float4 *>(mine + 16 * G::BN);
    for (int n = lane; n < G::BN; n += 32) sp4[n] = make_float4(0.f, 0.f, 0.f, 0.f);
    const uint32_t ntiles = *bt.ntiles;
    const float dt = (float)sp.dt, FLIP = (float)sp.FLIP;
    for (uint32_t q = box_next_tile(bt); q < ntiles; q = box_next_tile(bt)) {
        const uint32_t t = bt.tiles[q];
        int b0[3];
        box_tile_origin<D>(t, bt.sg, b0);
        b0[0] -= 1; b0[1] -= 1;
        if (D == 3) b0[2] -= 1;
        // gather box: as (second half of the record after the solve)
        for (int n = lane; n < G::BN; n += 32) {
            const int gi = box_global<G, D>(g, b0, n);
            ga[n] = gi >= 0 ? g.gat[gi].b : make_float4(0.f, 0.f, 0.f, 0.f);
        }
        const uint32_t k0 = t * 32u;
        const uint32_t cnt = bt.off[k0 + lane + 1] - bt.off[k0 + lane];
        uint32_t row = bt.off[k0];
        const uint32_t maxc = __reduce_max_sync(FULL, cnt);
        __syncwarp();
        for (uint32_t r = 0; r < maxc; ++r) {
            const bool act = cnt > r;
            const unsigned bal = __ballot_sync(FULL, act);
            const int64_t i = (int64_t)row + __popc(bal & lt);
            row += __popc(bal);
            AxisW<float> w[3];
            int lb[3] = {0, 0, 0};
            bool inside = false;
            float p[3] = {0, 0, 0};
            if (act) {
                double x[3];
                load_x<D, float>(P, i, x);
                float vo[3] = {0, 0, 0};
#pragma unroll
                for (int d = 0; d < D; ++d) vo[d] = ldcs(P.v[d] + i);
                const float m = ldcs(P.m + i);
                particle_weights<D, float>(x, g, w);
                float ta[3] = {0, 0, 0};
                inside = box_window<G, D>(w, b0, lb);
                if (inside) {
#pragma unroll
                    for (int c = 0; c < NC; ++c) {
                        const float wz = D == 3 ? w[2].N[c] : 1.0f;
#pragma unroll
                        for (int a = 0; a < 3; ++a) {
                            const int col = box_lin<G>(lb[0] + a, lb[1], lb[2] + (D == 3 ? c : 0));
                            float2 s01 = make_float2(0.f, 0.f);
                            float s2 = 0.f;
#pragma unroll
                            for (int b = 0; b < 3; ++b) {
                                const float wy = w[1].N[b];
                                const float4 q4 = ga[col + b];
                                s01 = __ffma2_rn(make_float2(wy, wy), make_float2(q4.x, q4.y), s01);
                                s2 += wy * q4.z;
                            }
                            const float wxz = w[0].N[a] * wz;
                            ta[0] += wxz * s01.x; ta[1] += wxz * s01.y; ta[2] += wxz * s2;
                        }
                    }
                } else {
                    const int n0 = window_n0<D, float>(g, w);
                    const int plane = g.nnx * g.nny;
#pragma unroll
                    for (int c = 0; c < NC; ++c) {
                        const float wz = D == 3 ? w[2].N[c] : 1.0f;
#pragma unroll
                        for (int a = 0; a < 3; ++a) {
                            const int col = n0 + a * g.nny + (D == 3 ? c * plane : 0);
                            float sa3[3] = {0, 0, 0};
#pragma unroll
                            for (int b = 0; b < 3; ++b) {
                                const float wy = w[1].N[b];
                                const float4 q4 = g.gat[col + b].b;
                                sa3[0] += wy * q4.x; sa3[1] += wy * q4.y; sa3[2] += wy * q4.z;
                            }
                            const float wxz = w[0].N[a] * wz;
#pragma unroll
                            for (int d = 0; d < 3; ++d) ta[d] += wxz * sa3[d];
                        }
                    }
                }
#pragma unroll
                for (int d = 0; d < D; ++d) {
                    const float vn = FLIP * vo[d] + ta[d] * dt;
                    stcs(P.v[d] + i, vn);
                    p[d] = m * vn;
                }
            }
            const int key = (act && inside) ? box_lin<G>(lb[0], lb[1], lb[2]) : -1 - lane;
            const unsigned same = __match_any_sync(FULL, key);
            const int grank = __popc(same & lt);
            const int rounds = __reduce_max_sync(FULL, (act && inside) ? grank : 0);
            for (int rr = 0; rr <= rounds; ++rr) {
                const bool mine = act && inside && grank == rr;
                const unsigned lanes = __ballot_sync(FULL, mine);
                if (mine) {
#pragma unroll
                    for (int c = 0; c < NC; ++c) {
                        const float wz = D == 3 ? w[2].N[c] : 1.0f;
#pragma unroll
                        for (int a = 0; a < 3; ++a) {
                            const float wxz = w[0].N[a] * wz;
                            const float2 P01 = make_float2(p[0] * wxz, p[1] * wxz);
                            const float P2 = p[2] * wxz;
                            const int col = box_lin<G>(lb[0] + a, lb[1], lb[2] + (D == 3 ? c : 0));
#pragma unroll
                            for (int b = 0; b < 3; ++b) {
                                const float wy = w[1].N[b];
                                const float4 A = sp4[col + b];
                                const float2 a01 = __ffma2_rn(make_float2(wy, wy), P01, make_float2(A.x, A.y));
                                sp4[col + b] = make_float4(a01.x, a01.y, fmaf(wy, P2, A.z), 0.f);
                                __syncwarp(lanes);
                            }
                        }
                    }
                }
                __syncwarp();
            }
            if (act && !inside) dm2_scatter<D, float>(g, w, p);
        }
        __syncwarp();
        for (int n = lane; n < G::BN; n += 32) {
            const float4 a = sp4[n];
            if (a.x != 0.f || a.y != 0.f || a.z != 0.f) {
                const int gi = box_global<G, D>(g, b0, n);
                if (gi >= 0) red_add4(&g.acc[gi].a, 0.f, a.x, a.y, a.z);
                sp4[n] = make_float4(0.f, 0.f, 0.f, 0.f);
            }
        }
        __syncwarp();
    }
}

}  // namespace mpm
