// mpm_kernels.cuh -- the kernels of one explicit uGIMP MUSL step.
//
// Step order of procedure!(…, Val(:OS), Val(:MUSL), Val(:a)),
// src/solvers/OS_MUSL.jl:58-102, mapped onto four launches:
//
//   k_solve      solvegrid_a_OS! / solvegrid_OS!   (nodes)     utils_OS.jl:507-640
//   k_dmap       doublemapping1(_a)_OS! + doublemapping2_OS!   utils_OS.jl:698-959
//   k_dm3        doublemapping3_OS!                (nodes)     utils_OS.jl:968-1016
//   k_g2p<FUSE>  G2P_OS! + liE! + dpP!/mcP!, and with FUSE the next step's
//                resetmpstatus_OS! + P2G_OS! at the new positions
//                                                   utils_OS.jl:178-496, 1025-1153
//
// resetgridstatus_OS! (utils_OS.jl:58-99) has no launch: the node passes clear
// the accumulators right after consuming them (k_solve clears momentum and
// force, k_dm3 clears mass and momentum), so the grid is zero again when the
// next P2G scatters.  Particle weights are recomputed from positions in each
// particle pass instead of being stored per particle.
//
// Node data are two records of one 32-byte sector each (FP32): the
// accumulator {m, px, py, pz | fx, fy, fz, 0} and the gather record
// {vsT, 0 | as, 0}, whose second half k_dm3 overwrites with Δus once the
// double mapping has consumed `as`.  Every particle-node touch therefore
// reads or reduces one sector.
#pragma once
#include "mpm_device.cuh"
#include "mpm_mc3d.cuh"

#include <climits>
#include <type_traits>

// resident CTAs of 256 threads per SM the particle passes are register-capped for
#ifndef MPM_P_MINB
#define MPM_P_MINB 4
#endif
// the double-mapping pass holds less state per particle: 6 CTAs (42 registers)
// measured faster than 4 for it, slower for the G2P pass
#ifndef MPM_DMAP_MINB
#define MPM_DMAP_MINB 6
#endif
// the lane-merged double mapping: 5 CTAs (48 registers) measured fastest
#ifndef MPM_DMAP_CHAIN_MINB
#define MPM_DMAP_CHAIN_MINB 5
#endif
// two-phase chain kernels (both phases' records): the fused pass measured
// 1.26 / 1.23 ms at 3 / 4 CTAs per SM on the 2.56 M saturated column, the
// double mapping 0.447 / 0.448 / 0.476 ms at 4 / 5 / 6
// the chain kernels in the all-FP64 mode: twice the registers per value; 3 CTAs
// (85 registers) measured 2.56 ms per step on the 2.56 M column against 2.63 at 2
#ifndef MPM_CHAIN_MINB_F64
#define MPM_CHAIN_MINB_F64 3
#endif
#ifndef MPM_TS_P_MINB
#define MPM_TS_P_MINB 4
#endif
// the two-phase fused pass in FP64: 2 CTAs (128 registers) ran 5.86 ms per step
// on the 2.56 M saturated column against 5.96 at 3
#ifndef MPM_TS_P_MINB_F64
#define MPM_TS_P_MINB_F64 2
#endif
#ifndef MPM_TS_DMAP_CHAIN_MINB
#define MPM_TS_DMAP_CHAIN_MINB 4
#endif

namespace mpm {

// Particle state, structure of arrays.  Positions are FP64 in every mode.
template <int D, typename R> struct PDev {
    static constexpr int NV = D == 2 ? 4 : 6;
    static constexpr int NF = D * D;
    double *x[3];
    R *v[3];
    R *sig[6];
    R *F[9];
    R *eps[6];
    R *epsq, *epsk, *epsv;
    R *m, *vol0, *vol;
    uint32_t *mat, *orig;
    R *coh;   // per-particle cohesion (random-field materials), else NULL
    // two-phase fields (coupling = :TS), else NULL: porosity n, pore pressure σw,
    // water mass mw = Ω·ρw (invariant like m), water velocity, water strain ϵijw
    R *n, *sigw, *mw;
    R *vw[3];
    R *epsw[6];
};

template <typename R> struct alignas(2 * sizeof(typename Vec<R>::T4)) Node8 {
    typename Vec<R>::T4 a, b;
};

template <typename R> struct GDev {
    using T4 = typename Vec<R>::T4;
    AxisC<R> ax[3];
    int nnx, nny, nnz;
    Node8<R> *acc;   // a = (m, px, py, pz), b = (fx, fy, fz, 0): P2G / DM2 accumulator
    Node8<R> *gat;   // a = (vsT, 0), b = (as, 0) after k_solve, (Δus, 0) after k_dm3
    T4 *gvs;         // vs (PIC != 0 or va = :v)
    const uint8_t *bcmask;  // bit d: velocity component d fixed
    const T4 *bcval;        // fixed values (NULL when all zero)
    const Mat<R> *mat;
    int *err;
    R *csigm, *comega;      // MVL: per-cell sum of vol*sigma_m and of vol (NULL when off)
    uint32_t *pcell;        // MVL: start-of-step cell of each particle
    uint32_t *bflag;        // per node block: 1 if some particle window touched it
    uint32_t *blist;        // the flagged blocks, in the order they were flagged
    uint32_t *bcount;       // number of entries in blist
    int nbx, nby, nbz;      // node blocks per axis (blocks of BX x BY x BZ nodes)
    // two-phase records (coupling = :TS), else NULL: acc holds {ms, ps | fs, mi}
    Node8<R> *accw;         // a = (mw, pw), b = (fw, 0)
    T4 *accd;               // drag force (fd, 0)
    Node8<R> *gatw;         // a = (vwT, 0), b = (vw, 0) after the solve, (Δuw, 0) after DM3
    const T4 *bcvalw;       // fixed water velocities (NULL when all zero); bcmask bits 3-5
};

// streaming (evict-first) access to the particle arrays, which are touched
// once per pass, so that the node records stay resident in L2
template <typename T> __device__ __forceinline__ T ldcs(const T *p) { return __ldcs(p); }
template <typename T> __device__ __forceinline__ void stcs(T *p, T v) { __stcs(p, v); }

// Node blocks: 4 (x) x 8 (y) x 4 (z) nodes in 3D, 8 (x) x 8 (y) in 2D; one
// CTA per block in the node passes (128 / 64 threads), y fastest.  The 2D
// blocks are the smaller because thin 2D bodies (slopes) leave more of a
// larger block's nodes massless; halving the 3D blocks measured slower.
template <int D> struct Blk {
    static constexpr int BX = D == 3 ? 4 : 8, BY = 8, BZ = D == 3 ? 4 : 1;
    static constexpr int NT = BX * BY * BZ;
};

template <int D, typename R> __device__ __forceinline__ void block_range(const GDev<R> &g, const AxisW<R> *w,
                                                                        int *lo, int *hi) {
    using B = Blk<D>;
    const int nn[3] = {g.nnx, g.nny, g.nnz};
    const int bs[3] = {B::BX, B::BY, B::BZ};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (a < D) {
            lo[a] = clampi(w[a].base, 0, nn[a] - 1) / bs[a];
            hi[a] = clampi(w[a].base + 2, 0, nn[a] - 1) / bs[a];
        } else {
            lo[a] = 0; hi[a] = 0;
        }
    }
}

// Flag node block b and append it to the active-block list the first time.
template <typename R> __device__ __forceinline__ void mark_block(const GDev<R> &g, int b) {
    if (g.bflag[b] == 0u && atomicExch(&g.bflag[b], 1u) == 0u) g.blist[atomicAdd(g.bcount, 1u)] = (uint32_t)b;
}

// Flag the node blocks covered by the windows of the calling lanes.  The
// active lanes of a warp (neighbouring particles after the cell sort) mark the
// bounding box of their windows together; a box wider than 64 blocks (lanes
// far apart) falls back to per-lane marking.  Marking is split in two: the
// flag exchanges are issued before the scatter (mark_begin) and their results
// are consumed after it (mark_end), so the atomics' round trip to L2 overlaps
// the reductions instead of stalling the warp.
struct MarkState {
    int b[2];
    unsigned old[2];
    int n;
};

template <int D, typename R>
__device__ __forceinline__ MarkState mark_begin(const GDev<R> &g, const AxisW<R> *w) {
    MarkState st;
    st.n = 0;
    int lo[3], hi[3];
    block_range<D, R>(g, w, lo, hi);
    const unsigned mask = __activemask();
    int blo[3], bhi[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        blo[a] = __reduce_min_sync(mask, lo[a]);
        bhi[a] = __reduce_max_sync(mask, hi[a]);
    }
    const int nx = bhi[0] - blo[0] + 1, ny = bhi[1] - blo[1] + 1, nz = bhi[2] - blo[2] + 1;
    const int total = nx * ny * nz;
    if (total <= 64) {
        const int lane = threadIdx.x & 31;
        const int rank = __popc(mask & ((1u << lane) - 1u)), cnt = __popc(mask);
        // decode k -> (by, bx, bz) without integer division: for k < 64 and box
        // sides <= 64, (k + 1/2)·(1/n) is at least 1/128 away from an integer,
        // far beyond the error of the approximate reciprocal
        const float rny = __fdividef(1.0f, (float)ny), rnx = __fdividef(1.0f, (float)nx);
        for (int k = rank; k < total; k += cnt) {
            const int r = __float2int_rz(((float)k + 0.5f) * rny);
            const int q = __float2int_rz(((float)r + 0.5f) * rnx);
            const int by = blo[1] + (k - r * ny), bx = blo[0] + (r - q * nx), bz = blo[2] + q;
            const int b = (bz * g.nbx + bx) * g.nby + by;
            if (st.n < 2) {
                st.b[st.n] = b;
                st.old[st.n] = atomicExch(&g.bflag[b], 1u);
                ++st.n;
            } else {
                mark_block<R>(g, b);
            }
        }
    } else {
        for (int bz = lo[2]; bz <= hi[2]; ++bz)
            for (int bx = lo[0]; bx <= hi[0]; ++bx)
                for (int by = lo[1]; by <= hi[1]; ++by) {
                    mark_block<R>(g, (bz * g.nbx + bx) * g.nby + by);
                }
    }
    return st;
}

// append the blocks this lane flagged first to the active-block list
template <typename R> __device__ __forceinline__ void mark_end(const GDev<R> &g, const MarkState &st) {
#pragma unroll
    for (int j = 0; j < 2; ++j)
        if (j < st.n && st.old[j] == 0u) g.blist[atomicAdd(g.bcount, 1u)] = (uint32_t)st.b[j];
}

// node of thread t in block b (returns -1 outside the grid)
template <int D, typename R> __device__ __forceinline__ int block_node(const GDev<R> &g, int b, int t) {
    using B = Blk<D>;
    int by = b % g.nby;
    int r = b / g.nby;
    int bx = r % g.nbx;
    int bz = r / g.nbx;
    int ly = t % B::BY, lx = (t / B::BY) % B::BX, lz = t / (B::BY * B::BX);
    int ix = bx * B::BX + lx, iy = by * B::BY + ly, iz = bz * B::BZ + lz;
    if (ix >= g.nnx || iy >= g.nny || (D == 3 && iz >= g.nnz)) return -1;
    return D == 2 ? ix * g.nny + iy : (iz * g.nnx + ix) * g.nny + iy;
}

// Stress-return surrogate hooks of the particle pass (3D Drucker-Prager).
//   mode 1: run the plain return and log a sample of the yielding particles
//           (features: trial stress 6, strain increment 6, plastic strain,
//           cohesion, friction; target: returned stress 6);
//   mode 2: defer every yielding particle: keep its trial stress, write its
//           features and index to the work list (the surrogate and the
//           fallback finish them before the scatter).
struct SurrCtx {
    int mode;
    uint32_t every, salt;   // mode 1: keep a yielding particle if hash(i, salt) % every == 0
    uint32_t cap;           // rows of feat / tgt / list
    float *feat;            // cap x 16
    float *tgt;             // cap x 6 (mode 1)
    uint32_t *cnt;          // rows written (may exceed cap: extra rows are dropped)
    uint32_t *list;         // mode 2: particle index of each row
};

struct StepParams {
    double dt;
    double G;        // gravity of the scatter (P2G) in this launch
    double FLIP, PIC, zeta;
    int plastic;     // Ti >= Te
    int constitutive;
    int va;          // 0 = :a, 1 = :v
    int need_vs;     // DM gathers grid vs
    int mc3d;        // 3D Mohr-Coulomb: 0 elastic predictor only (literal), 1 restated return
    int mvl;         // volumetric-locking mitigation (cell-averaged mean stress)
    int usl;         // USL scheme (OS_USL.jl): no double mapping, Δu = vsT·dt
    int prefetch;    // FP32 particle pass: fields staged in dynamic shared memory (PF_N x 256 floats)
    int ts;          // two-phase coupling (TS_MUSL.jl)
    double zeta_w;   // ζw, water damping (two-phase)
    double meps;     // nodal mass below which a node is massless: eps of the reference's float type
    SurrCtx surr;
    int64_t np;
};

template <int D> __device__ __forceinline__ int node_id(int ix, int iy, int iz, int nnx, int nny) {
    return D == 2 ? ix * nny + iy : (iz * nnx + ix) * nny + iy;
}

// Cell of a particle per axis (0-based), Julia rule: x and z by fld, y by cld
// (utils_OS.jl:247-249, 380-383).
template <int D, typename R>
__device__ __forceinline__ void particle_cell(const double *xp, const GDev<R> &g, int *ci) {
    ci[0] = cell_fld<R>(xp[0], g.ax[0]);
    ci[1] = cell_cld_m1<R>(xp[1], g.ax[1]);
    if (D == 3) ci[2] = cell_fld<R>(xp[2], g.ax[2]);
}

// Weights of the 3^D window of a particle.  Returns false if the particle is
// out of the grid (its contributions are then dropped and the flag raised).
//
// FP32 mode takes a short cut for windows inside the grid: the window corner
// is node ci - 1 below the cell centre and ci above it (axis_weights), i.e.
// node floor(t - 1/2) with t = (ξ - x1)/h, whichever of Julia's fld / cld the
// cell index uses (they differ only at t integral, where both give that node);
// the distances to the three nodes are then s - k·h with s = ξ - x_corner.  At
// t - 1/2 integral (a particle exactly at a cell centre) the two candidate
// windows differ only by a node of weight 0.  Windows that touch the grid's
// last node layer, and non-finite positions, take the general path below.
template <int D, typename R>
__device__ __forceinline__ bool particle_weights(const double *xp, const GDev<R> &g, AxisW<R> *w) {
    if constexpr (sizeof(R) == 4) {
        bool inner = true;
        double sd[3];
        int bs[3];
#pragma unroll
        for (int a = 0; a < D; ++a) {
            const double t = (xp[a] - g.ax[a].x1) * g.ax[a].inv_h - 0.5;
            const double f = floor(t);
            inner = inner && f >= 0.0 && f + 2.0 < (double)g.ax[a].nn;   // false for NaN
            bs[a] = inner ? (int)f : 0;
            sd[a] = xp[a] - (g.ax[a].x1 + (double)bs[a] * g.ax[a].h);
        }
        if (inner) {
#pragma unroll
            for (int a = 0; a < D; ++a) {
                const float sf = (float)sd[a];
                w[a].base = bs[a];
#pragma unroll
                for (int k = 0; k < 3; ++k) ugimp1<R>(sf - (float)k * g.ax[a].hr, g.ax[a], w[a].N[k], w[a].dN[k]);
            }
            if (D == 2) w[2].base = 0;
            return true;
        }
    }
    int ci[3];
    particle_cell<D, R>(xp, g, ci);
    bool bad = false;
#pragma unroll
    for (int a = 0; a < D; ++a) {
        int c = ci[a];
        if (c < 0 || c >= g.ax[a].nc) { bad = true; c = clampi(c, 0, g.ax[a].nc - 1); }
        if (axis_weights<R>(xp[a], c, g.ax[a], w[a])) bad = true;
    }
    if (D == 2) w[2].base = 0;
    if (bad) {
        // out-of-grid particle: no weight, and a window at the grid origin so
        // that any address formed from it stays inside the node arrays
#pragma unroll
        for (int a = 0; a < D; ++a) {
            w[a].base = 0;
#pragma unroll
            for (int k = 0; k < 3; ++k) { w[a].N[k] = R(0); w[a].dN[k] = R(0); }
        }
    }
    return !bad;
}

// node index of the window corner; window node (a, b, c) is
// n0 + a*nny + b + c*nnx*nny (3D) / n0 + a*nny + b (2D)
template <int D, typename R> __device__ __forceinline__ int window_n0(const GDev<R> &g, const AxisW<R> *w) {
    return D == 2 ? w[0].base * g.nny + w[1].base : (w[2].base * g.nnx + w[0].base) * g.nny + w[1].base;
}

template <int D, typename R>
__device__ __forceinline__ int window_node(const GDev<R> &g, const AxisW<R> *w, int a, int b, int c) {
    return window_n0<D, R>(g, w) + a * g.nny + b + (D == 3 ? c * g.nnx * g.nny : 0);
}

// ---------------------------------------------------------------------------
// P2G scatter of one particle (P2G_OS!, utils_OS.jl:424-496): nodal mass,
// momentum and force; gravity on the last axis.  Nodes with N == 0 are skipped
// like the reference's `if Ni ≠ 0`.
//
// The weights are separable, N = Nx·Ny·Nz and ∇N = (dNx·Ny·Nz, Nx·dNy·Nz,
// Nx·Ny·dNz), so the terms that do not depend on the y index are formed once
// per (x, z) column of the window: with σv = -Ω·σ,
//   f_k(node) = Ny·X_k + dNy·Y_k,  X_k = σv_kx·dNx·Nz + σv_kz·Nx·dNz (+ m·Nx·Nz·g
//   on the gravity axis), Y_k = σv_ky·Nx·Nz;  m·N = Ny·(m·Nx·Nz), p·N likewise.
// ---------------------------------------------------------------------------
template <int D, typename R>
__device__ __forceinline__ void p2g_scatter(const GDev<R> &g, const AxisW<R> *w, R m, R vol,
                                            const R *v, const R *s, R G) {
    const MarkState mk = mark_begin<D, R>(g, w);
    const R p[3] = {m * v[0], m * v[1], D == 3 ? m * v[2] : R(0)};
    const int n0 = window_n0<D, R>(g, w);
    const int plane = g.nnx * g.nny;
    if (D == 2) {
        // σv rows: (xx, xy), (xy, yy)
        const R sxx = -vol * s[0], syy = -vol * s[1], sxy = -vol * s[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const R wx = w[0].N[a], gx = w[0].dN[a];
            if (wx == R(0)) continue;
            const R M = m * wx, P0 = p[0] * wx, P1 = p[1] * wx;
            const R X0 = sxx * gx, X1 = sxy * gx + M * G;
            const R Y0 = sxy * wx, Y1 = syy * wx;
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                const R wy = w[1].N[b], gy = w[1].dN[b];
                if (wy == R(0)) continue;
                Node8<R> *q = g.acc + (n0 + a * g.nny + b);
                red_add4(&q->a, M * wy, P0 * wy, P1 * wy, R(0));
                red_add4(&q->b, wy * X0 + gy * Y0, wy * X1 + gy * Y1, R(0), R(0));
            }
        }
    } else {
        const R sv[6] = {-vol * s[0], -vol * s[1], -vol * s[2], -vol * s[3], -vol * s[4], -vol * s[5]};
        // Voigt xx yy zz xy yz zx: rows x = (0, 3, 5), y = (3, 1, 4), z = (5, 4, 2)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const R wz = w[2].N[c], gz = w[2].dN[c];
            if (wz == R(0)) continue;
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const R wx = w[0].N[a];
                if (wx == R(0)) continue;
                const R wxz = wx * wz, gxz = w[0].dN[a] * wz, xdz = wx * gz;
                const R M = m * wxz, P0 = p[0] * wxz, P1 = p[1] * wxz, P2 = p[2] * wxz;
                const R X0 = sv[0] * gxz + sv[5] * xdz;
                const R X1 = sv[3] * gxz + sv[4] * xdz;
                const R X2 = sv[5] * gxz + sv[2] * xdz + M * G;
                const R Y0 = sv[3] * wxz, Y1 = sv[1] * wxz, Y2 = sv[4] * wxz;
                Node8<R> *col = g.acc + (n0 + a * g.nny + c * plane);
#pragma unroll
                for (int b = 0; b < 3; ++b) {
                    const R wy = w[1].N[b], gy = w[1].dN[b];
                    if (wy == R(0)) continue;
                    red_add4(&col[b].a, M * wy, P0 * wy, P1 * wy, P2 * wy);
                    red_add4(&col[b].b, wy * X0 + gy * Y0, wy * X1 + gy * Y1, wy * X2 + gy * Y2, R(0));
                }
            }
        }
    }
    mark_end<R>(g, mk);
}

template <int D, typename R>
__device__ __forceinline__ void load_x(const PDev<D, R> &P, int64_t i, double *x) {
    x[0] = ldcs(P.x[0] + i); x[1] = ldcs(P.x[1] + i);
    x[2] = D == 3 ? ldcs(P.x[2] + i) : 0.0;
}

// Standalone P2G (first step after an upload; per-stage checks).
template <int D, typename R>
__global__ void __launch_bounds__(256) k_p2g(PDev<D, R> P, GDev<R> g, StepParams sp) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= sp.np) return;
    double x[3];
    load_x<D, R>(P, i, x);
    AxisW<R> w[3];
    if (!particle_weights<D, R>(x, g, w)) { atomicOr(g.err, ERR_OOG); return; }
    R v[3] = {P.v[0][i], P.v[1][i], D == 3 ? P.v[2][i] : R(0)};
    R s[6];
#pragma unroll
    for (int k = 0; k < PDev<D, R>::NV; ++k) s[k] = P.sig[k][i];
    p2g_scatter<D, R>(g, w, P.m[i], P.vol[i], v, s, (R)sp.G);
}

// ---------------------------------------------------------------------------
// Grid solve: solvegrid_a_OS! (va = :a, utils_OS.jl:547-640) or solvegrid_OS!
// (va = :v, utils_OS.jl:507-535, 650-687).  Clears momentum and force.
// ---------------------------------------------------------------------------
template <int D, typename R>
__device__ __forceinline__ void solve_node(const GDev<R> &g, const StepParams &sp, int i) {
    using T4 = typename Vec<R>::T4;
    Node8<R> A = g.acc[i];
    const T4 a0 = A.a, a1 = A.b;
    if (a0.x == R(0) && a0.y == R(0) && a0.z == R(0) && a0.w == R(0) && a1.x == R(0) && a1.y == R(0) &&
        a1.z == R(0)) {
        // untouched node: every derived quantity is 0 (ms_denom = 0); the BC
        // can only write its value, which is 0 unless bcval is present.
        if (g.bcval == nullptr || g.bcmask[i] == 0) {
            Node8<R> z;
            z.a = mk4<R>(0, 0, 0, 0);
            z.b = z.a;
            g.gat[i] = z;
            if (sp.need_vs) g.gvs[i] = z.a;
            return;
        }
    }
    const R eps = (R)sp.meps;
    R m = a0.x;
    R md = m < eps ? R(0) : R(1) / m;
    R p[3] = {a0.y, a0.z, a0.w};
    R f[3] = {a1.x, a1.y, a1.z};
    uint8_t bm = g.bcmask[i];
    R bv[3] = {R(0), R(0), R(0)};
    if (g.bcval) { T4 b = g.bcval[i]; bv[0] = b.x; bv[1] = b.y; bv[2] = b.z; }
    const R dt = (R)sp.dt;
    R vs[3], vT[3], as[3];
    R ss = R(0);
#pragma unroll
    for (int d = 0; d < D; ++d) ss += f[d] * f[d];
    R damp = -(R)sp.zeta * sqrt(ss);
    if (sp.va == 0) {
#pragma unroll
        for (int d = 0; d < D; ++d) {
            if (bm & (1 << d)) p[d] = bv[d];
            vs[d] = p[d] * md;
            R Fs = f[d] + damp * sgn(vs[d]);
            vT[d] = vs[d] + Fs * dt * md;
            as[d] = Fs * md;
            if (bm & (1 << d)) { vT[d] = bv[d]; as[d] = bv[d]; }
        }
    } else {
#pragma unroll
        for (int d = 0; d < D; ++d) {
            vs[d] = p[d] * md;
            R Fs = f[d] + damp * sgn(vs[d]);
            vT[d] = (p[d] + Fs * dt) * md;
            as[d] = R(0);
            if (bm & (1 << d)) vT[d] = bv[d];
        }
    }
    if (D == 2) { vs[2] = vT[2] = as[2] = R(0); }
    Node8<R> G;
    G.a = mk4<R>(vT[0], vT[1], vT[2], 0);
    G.b = mk4<R>(as[0], as[1], as[2], 0);
    g.gat[i] = G;
    if (sp.need_vs) g.gvs[i] = mk4<R>(vs[0], vs[1], vs[2], 0);
    A.a = mk4<R>(sp.usl ? R(0) : m, 0, 0, 0);   // MUSL keeps m for DM3
    A.b = mk4<R>(0, 0, 0, 0);
    g.acc[i] = A;
}

// One CTA per active node block, grid-stride over the active-block list.
template <int D, typename R>
__global__ void __launch_bounds__(128) k_solve(GDev<R> g, StepParams sp) {
    const uint32_t n = *g.bcount;
    for (uint32_t k = blockIdx.x; k < n; k += gridDim.x) {
        const int b = (int)g.blist[k];
        const int i = block_node<D, R>(g, b, threadIdx.x);
        if (i >= 0) solve_node<D, R>(g, sp, i);
        if (sp.usl && threadIdx.x == 0) g.bflag[b] = 0u;   // USL has no DM3 to clear it
    }
}

// ---------------------------------------------------------------------------
// Warp-level merging of the scatters (FP32).  After the cell sort the lanes of
// a warp hold the particles of equal rank in consecutive cells of a tile, y
// fastest, so lane L's window usually starts one node above lane L-1's in y
// with the same x and z (a "chain" of up to 8 lanes).  Then the node at
// window row b = 0 of lane L is also row 1 of lane L-1 and row 2 of lane L-2:
// lane L adds those two contributions (shuffled up) to its own and reduces
// the sum into global memory once, and only the last lane of a chain also
// reduces rows 1 and 2.  A chain of 8 lanes issues 10 node reductions per
// (x, z) window column instead of 24.  Lanes that are not chained (any other
// window offset, dead or out-of-grid lanes) simply emit all three rows.  All
// 32 lanes of the warp must call these functions.
// ---------------------------------------------------------------------------
// chain key of a lane without a particle: never one more than another key
__device__ __forceinline__ int dead_key() { return -(1 << 30) - 4 * (int)(threadIdx.x & 31); }

struct Chain {
    bool c1;    // lane L-1's window is this window shifted by -1 in y
    bool c2;    // ... and lane L-2's by -2
    bool end;   // lane L+1 does not continue the chain
    bool x1;    // lane L-8's window is this window shifted by -1 in x
    bool x2;    // ... and lane L-16's by -2
    bool xend;  // lane L+8 does not continue the x chain
};

// nny = nodes along y: the x step of a window corner
__device__ __forceinline__ Chain chain_of(int n0, int nny) {
    const int lane = threadIdx.x & 31;
    const unsigned F = 0xffffffffu;
    const int p1 = __shfl_up_sync(F, n0, 1), p2 = __shfl_up_sync(F, n0, 2);
    const int q1 = __shfl_down_sync(F, n0, 1);
    const int r1 = __shfl_up_sync(F, n0, 8), r2 = __shfl_up_sync(F, n0, 16);
    const int s1 = __shfl_down_sync(F, n0, 8);
    Chain c;
    c.c1 = lane >= 1 && p1 == n0 - 1;
    c.c2 = c.c1 && lane >= 2 && p2 == n0 - 2;
    c.end = !(lane <= 30 && q1 == n0 + 1);
    c.x1 = lane >= 8 && r1 == n0 - nny;
    c.x2 = c.x1 && lane >= 16 && r2 == n0 - 2 * nny;
    c.xend = !(lane < 24 && s1 == n0 + nny);
    return c;
}

// Merge of row 0 across x: the three window columns a = 0, 1, 2 of row 0 (already
// merged along y) of lane L are columns 1 and 2 of lanes L-8 and L-16 when those
// lanes sit one and two cells lower in x (the cell order of a tile puts 8 cells
// along y, so lane L-8 holds the same rank in the x-neighbouring cell).  Column
// 0 takes the two shuffled contributions; only the last lane of an x chain also
// emits columns 1 and 2.  v[a][k]: k-th component of column a; returns whether
// column a is emitted by this lane.
template <typename R, int K>
__device__ __forceinline__ void xmerge_row0(const Chain &ch, R (*v)[K], bool *emit) {
    const unsigned F = 0xffffffffu;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const R a1 = __shfl_up_sync(F, v[1][k], 8), a2 = __shfl_up_sync(F, v[2][k], 16);
        const R b2 = __shfl_up_sync(F, v[2][k], 8);
        v[0][k] += (ch.x1 ? a1 : R(0.0)) + (ch.x2 ? a2 : R(0.0));
        v[1][k] += ch.x1 ? b2 : R(0.0);
    }
    emit[0] = true;
    emit[1] = emit[2] = ch.xend;
}

// doublemapping2 (momentum N·p) with chained lanes merged; n0 = window corner,
// key = n0 for a live lane, a value no other lane's key follows for a dead one
template <int D, typename R = float>
__device__ __forceinline__ void dm2_scatter_chain(const GDev<R> &g, const AxisW<R> *w, int n0, int key,
                                                  const R *p) {
    const Chain ch = chain_of(key, g.nny);
    const unsigned F = 0xffffffffu;
    R p1[3], p2[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        p1[k] = __shfl_up_sync(F, p[k], 1);
        p2[k] = __shfl_up_sync(F, p[k], 2);
    }
    const int plane = g.nnx * g.nny;
    constexpr int NC = D == 3 ? 3 : 1;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        const R wz = D == 3 ? w[2].N[c] : R(1.0);
        R r0[3][3];   // row 0 of columns a = 0..2 (merged along y)
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const R wxz = w[0].N[a] * wz;
            const R N0 = wxz * w[1].N[0], N1 = wxz * w[1].N[1], N2 = wxz * w[1].N[2];
            const R u1 = __shfl_up_sync(F, N1, 1), u2 = __shfl_up_sync(F, N2, 2), v2 = __shfl_up_sync(F, N2, 1);
            const R a1 = ch.c1 ? u1 : R(0.0), a2 = ch.c2 ? u2 : R(0.0), b2 = ch.c1 ? v2 : R(0.0);
#pragma unroll
            for (int k = 0; k < 3; ++k) r0[a][k] = N0 * p[k] + a1 * p1[k] + a2 * p2[k];
            // rows 1 and 2 by the chain's last lane (predicated, not branched)
            Node8<R> *col = g.acc + (n0 + a * g.nny + c * plane);
            red_add4_if(ch.end && N1 + b2 != R(0.0), &col[1].a, R(0.0), N1 * p[0] + b2 * p1[0],
                        N1 * p[1] + b2 * p1[1], N1 * p[2] + b2 * p1[2]);
            red_add4_if(ch.end && N2 != R(0.0), &col[2].a, R(0.0), N2 * p[0], N2 * p[1], N2 * p[2]);
        }
        bool emit[3];
        xmerge_row0<R, 3>(ch, r0, emit);
#pragma unroll
        for (int a = 0; a < 3; ++a)
            red_add4_if(emit[a] && (r0[a][0] != R(0.0) || r0[a][1] != R(0.0) || r0[a][2] != R(0.0)),
                        &g.acc[n0 + a * g.nny + c * plane].a, R(0.0), r0[a][0], r0[a][1], r0[a][2]);
    }
}

// One N-proportional record (node value N·V, V a lane constant of K <= 4
// components) scattered with chained lanes merged: row 0 of a window column
// takes lane L-1's row 1 and lane L-2's row 2 (V and the weights shuffled);
// rows 1 and 2 are reduced by the chain's last lane.  rec(i) is the record of
// node i.  All lanes call it.
template <int D, int K, typename R, typename Rec>
__device__ __forceinline__ void chain_nprop(const GDev<R> &g, const AxisW<R> *w, int n0, const Chain &ch,
                                               const R *V, Rec rec) {
    const unsigned F = 0xffffffffu;
    R V1[K], V2[K];
#pragma unroll
    for (int k = 0; k < K; ++k) { V1[k] = __shfl_up_sync(F, V[k], 1); V2[k] = __shfl_up_sync(F, V[k], 2); }
    const int plane = g.nnx * g.nny;
    constexpr int NC = D == 3 ? 3 : 1;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        const R wz = D == 3 ? w[2].N[c] : R(1.0);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const R wx = w[0].N[a];
            const int col = n0 + a * g.nny + c * plane;
            const R N0 = wx * w[1].N[0] * wz, N1 = wx * w[1].N[1] * wz, N2 = wx * w[1].N[2] * wz;
            const R u1 = __shfl_up_sync(F, N1, 1), u2 = __shfl_up_sync(F, N2, 2);
            const R v2 = __shfl_up_sync(F, N2, 1);
            const R f1 = ch.c1 ? u1 : R(0.0), f2 = ch.c2 ? u2 : R(0.0), e1 = ch.c1 ? v2 : R(0.0);
            R r[4] = {R(0.0), R(0.0), R(0.0), R(0.0)};
            if (N0 + f1 + f2 != R(0.0)) {
#pragma unroll
                for (int k = 0; k < K; ++k) r[k] = N0 * V[k] + f1 * V1[k] + f2 * V2[k];
                red_add4(rec(col), r[0], r[1], r[2], r[3]);
            }
            if (ch.end) {
                if (N1 + e1 != R(0.0)) {
#pragma unroll
                    for (int k = 0; k < K; ++k) r[k] = N1 * V[k] + e1 * V1[k];
                    red_add4(rec(col + 1), r[0], r[1], r[2], r[3]);
                }
                if (N2 != R(0.0)) {
#pragma unroll
                    for (int k = 0; k < K; ++k) r[k] = N2 * V[k];
                    red_add4(rec(col + 2), r[0], r[1], r[2], r[3]);
                }
            }
        }
    }
}

// P2G_OS! of one particle with chained lanes merged (the arithmetic of
// p2g_scatter; 7 components per node: m, p, f)
template <int D, typename R = float>
__device__ __forceinline__ void p2g_scatter_chain(const GDev<R> &g, const AxisW<R> *w, int n0, int key,
                                                  R m, R vol, const R *v, const R *s, R G) {
    if constexpr (std::is_same<R, float>::value) {
        const Chain ch = chain_of(key, g.nny);
        const unsigned F = 0xffffffffu;
        const float p[3] = {m * v[0], m * v[1], D == 3 ? m * v[2] : 0.0f};
        const int plane = g.nnx * g.nny;
        constexpr int NC = D == 3 ? 3 : 1;
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
                // per column: node value = Ny·(M, P, X) + dNy·(0, 0, Y)
                float U[7], Y[3];
                U[0] = m * wxz;
                U[1] = p[0] * wxz; U[2] = p[1] * wxz; U[3] = p[2] * wxz;
                if (D == 2) {
                    U[4] = sv[0] * gxz; U[5] = sv[3] * gxz + U[0] * G; U[6] = 0.0f;
                    Y[0] = sv[3] * wxz; Y[1] = sv[1] * wxz; Y[2] = 0.0f;
                } else {
                    U[4] = sv[0] * gxz + sv[5] * xdz;
                    U[5] = sv[3] * gxz + sv[4] * xdz;
                    U[6] = sv[5] * gxz + sv[2] * xdz + U[0] * G;
                    Y[0] = sv[3] * wxz; Y[1] = sv[1] * wxz; Y[2] = sv[4] * wxz;
                }
                // this lane's rows b = 0, 1, 2 as component pairs (packed FP32 arithmetic):
                // (m, px), (py, pz), (fx, fy), (fz, 0)
                float2 r0[4], r1[4], r2[4];
                const float2 U01 = make_float2(U[0], U[1]), U23 = make_float2(U[2], U[3]);
                const float2 U45 = make_float2(U[4], U[5]), Y01 = make_float2(Y[0], Y[1]);
#pragma unroll
                for (int b = 0; b < 3; ++b) {
                    const float wy = w[1].N[b], gy = w[1].dN[b];
                    const float2 w2 = make_float2(wy, wy), g2 = make_float2(gy, gy);
                    float2 *r = b == 0 ? r0 : (b == 1 ? r1 : r2);
                    r[0] = __fmul2_rn(w2, U01);
                    r[1] = __fmul2_rn(w2, U23);
                    r[2] = __ffma2_rn(w2, U45, __fmul2_rn(g2, Y01));
                    r[3] = make_float2(wy * U[6] + gy * Y[2], 0.0f);
                }
                // row 0 += lane L-1's row 1 + lane L-2's row 2; chain ends: row 1 += lane L-1's row 2
                const float f1 = ch.c1 ? 1.0f : 0.0f, f2 = ch.c2 ? 1.0f : 0.0f;
                const float2 c1 = make_float2(f1, f1), c2 = make_float2(f2, f2);
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const float2 x1 = make_float2(__shfl_up_sync(F, r1[j].x, 1), __shfl_up_sync(F, r1[j].y, 1));
                    const float2 x2 = make_float2(__shfl_up_sync(F, r2[j].x, 2), __shfl_up_sync(F, r2[j].y, 2));
                    const float2 y2 = make_float2(__shfl_up_sync(F, r2[j].x, 1), __shfl_up_sync(F, r2[j].y, 1));
                    r0[j] = __ffma2_rn(c2, x2, __ffma2_rn(c1, x1, r0[j]));
                    r1[j] = __ffma2_rn(c1, y2, r1[j]);
                }
                Node8<float> *col = g.acc + (n0 + a * g.nny + c * plane);
                if (r0[0].x != 0.0f) {
                    red_add4(&col[0].a, r0[0].x, r0[0].y, r0[1].x, r0[1].y);
                    red_add4(&col[0].b, r0[2].x, r0[2].y, r0[3].x, 0.0f);
                }
                if (ch.end) {
                    if (r1[0].x != 0.0f) {
                        red_add4(&col[1].a, r1[0].x, r1[0].y, r1[1].x, r1[1].y);
                        red_add4(&col[1].b, r1[2].x, r1[2].y, r1[3].x, 0.0f);
                    }
                    if (r2[0].x != 0.0f) {
                        red_add4(&col[2].a, r2[0].x, r2[0].y, r2[1].x, r2[1].y);
                        red_add4(&col[2].b, r2[2].x, r2[2].y, r2[3].x, 0.0f);
                    }
                }
            }
        }

    } else {
        // FP64: the same rows and merging, component by component
        const Chain ch = chain_of(key, g.nny);
        const unsigned F = 0xffffffffu;
        const R p[3] = {m * v[0], m * v[1], D == 3 ? m * v[2] : R(0)};
        const int plane = g.nnx * g.nny;
        constexpr int NC = D == 3 ? 3 : 1;
        R sv[6];
        if (D == 2) {
            sv[0] = -vol * s[0]; sv[1] = -vol * s[1]; sv[3] = -vol * s[3];
            sv[2] = sv[4] = sv[5] = R(0);
        } else {
#pragma unroll
            for (int k = 0; k < 6; ++k) sv[k] = -vol * s[k];
        }
        const R f1 = ch.c1 ? R(1) : R(0), f2 = ch.c2 ? R(1) : R(0);
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            const R wz = D == 3 ? w[2].N[c] : R(1), gz = D == 3 ? w[2].dN[c] : R(0);
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const R wx = w[0].N[a];
                const R wxz = wx * wz, gxz = w[0].dN[a] * wz, xdz = wx * gz;
                R U[7], Y[3];
                U[0] = m * wxz;
                U[1] = p[0] * wxz; U[2] = p[1] * wxz; U[3] = p[2] * wxz;
                if (D == 2) {
                    U[4] = sv[0] * gxz; U[5] = sv[3] * gxz + U[0] * G; U[6] = R(0);
                    Y[0] = sv[3] * wxz; Y[1] = sv[1] * wxz; Y[2] = R(0);
                } else {
                    U[4] = sv[0] * gxz + sv[5] * xdz;
                    U[5] = sv[3] * gxz + sv[4] * xdz;
                    U[6] = sv[5] * gxz + sv[2] * xdz + U[0] * G;
                    Y[0] = sv[3] * wxz; Y[1] = sv[1] * wxz; Y[2] = sv[4] * wxz;
                }
                // rows b = 0, 1, 2: (m, px, py, pz, fx, fy, fz)
                R r[3][7];
#pragma unroll
                for (int b = 0; b < 3; ++b) {
                    const R wy = w[1].N[b], gy = w[1].dN[b];
#pragma unroll
                    for (int k = 0; k < 4; ++k) r[b][k] = wy * U[k];
#pragma unroll
                    for (int k = 0; k < 3; ++k) r[b][4 + k] = wy * U[4 + k] + gy * Y[k];
                }
#pragma unroll
                for (int j = 0; j < 7; ++j) {
                    const R x1 = __shfl_up_sync(F, r[1][j], 1), x2 = __shfl_up_sync(F, r[2][j], 2);
                    const R y2 = __shfl_up_sync(F, r[2][j], 1);
                    r[0][j] += f1 * x1 + f2 * x2;
                    r[1][j] += f1 * y2;
                }
                Node8<R> *col = g.acc + (n0 + a * g.nny + c * plane);
#pragma unroll
                for (int b = 0; b < 3; ++b) {
                    if (b > 0 && !ch.end) break;
                    if (r[b][0] == R(0)) continue;
                    red_add4(&col[b].a, r[b][0], r[b][1], r[b][2], r[b][3]);
                    red_add4(&col[b].b, r[b][4], r[b][5], r[b][6], R(0));
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Double mapping: doublemapping1_a_OS! / doublemapping1_OS! (new particle
// velocity from the grid) fused with doublemapping2_OS! (re-scatter of the
// particle momentum with the same weights).  The position update of DM1 is
// carried out by k_g2p, which gathers the same ΣN·vsT with the same weights.
// ---------------------------------------------------------------------------
// doublemapping1 of one particle: gathers, new velocity (stored), momentum p
// for the re-scatter; w receives the particle's window.
// GEN = false: the va = :a scheme without the separate grid velocity (the
// common case), with the two run-time gather switches folded away.
template <int D, typename R, bool GEN = true>
__device__ __forceinline__ void dmap_core(const PDev<D, R> &P, const GDev<R> &g, const StepParams &sp, int64_t i,
                                          AxisW<R> *w, R *p) {
    using T4 = typename Vec<R>::T4;
    double x[3];
    load_x<D, R>(P, i, x);
    R vo[3];
#pragma unroll
    for (int d = 0; d < D; ++d) vo[d] = ldcs(P.v[d] + i);
    const R m = ldcs(P.m + i);
    particle_weights<D, R>(x, g, w);   // out-of-grid particles get zero weights
    const int n0 = window_n0<D, R>(g, w);
    const int plane = g.nnx * g.nny;
    R tT[3] = {0, 0, 0}, ta[3] = {0, 0, 0}, tv[3] = {0, 0, 0};
    constexpr int NC = D == 3 ? 3 : 1;
    const bool va_v = GEN && sp.va != 0, need_vs = GEN && sp.need_vs != 0;
    // ΣN·q = Σ_(x,z) Nx·Nz·(Σ_y Ny·q): inner sums along the contiguous y run
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        const R wz = D == 3 ? w[2].N[c] : R(1);
        if (wz == R(0)) continue;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const R wx = w[0].N[a];
            if (wx == R(0)) continue;
            const int col = n0 + a * g.nny + c * plane;
            R sT[3] = {0, 0, 0}, sa[3] = {0, 0, 0}, sv[3] = {0, 0, 0};
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                const R wy = w[1].N[b];
                if (wy == R(0)) continue;
                const T4 qb = g.gat[col + b].b;   // every valid window lies inside the grid
                sa[0] += wy * qb.x; sa[1] += wy * qb.y; sa[2] += wy * qb.z;
                if (va_v) {
                    const T4 qa = g.gat[col + b].a;
                    sT[0] += wy * qa.x; sT[1] += wy * qa.y; sT[2] += wy * qa.z;
                }
                if (need_vs) {
                    const T4 vs = g.gvs[col + b];
                    sv[0] += wy * vs.x; sv[1] += wy * vs.y; sv[2] += wy * vs.z;
                }
            }
            const R wxz = wx * wz;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                ta[d] += wxz * sa[d];
                tT[d] += wxz * sT[d];
                tv[d] += wxz * sv[d];
            }
        }
    }
    const R dt = (R)sp.dt, FLIP = (R)sp.FLIP, PIC = (R)sp.PIC;
    R vn[3] = {0, 0, 0};
#pragma unroll
    for (int d = 0; d < D; ++d) {
        if (!va_v) vn[d] = FLIP * vo[d] + PIC * tv[d] + ta[d] * dt;
        else vn[d] = FLIP * (vo[d] + (tT[d] - tv[d])) + PIC * tT[d];
        stcs(P.v[d] + i, vn[d]);
    }
    p[0] = m * vn[0]; p[1] = m * vn[1]; p[2] = D == 3 ? m * vn[2] : R(0);
}

// doublemapping2 of one particle: p·N into the momentum of the window nodes
template <int D, typename R>
__device__ __forceinline__ void dm2_scatter(const GDev<R> &g, const AxisW<R> *w, const R *p) {
    const int n0 = window_n0<D, R>(g, w);
    const int plane = g.nnx * g.nny;
    constexpr int NC = D == 3 ? 3 : 1;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        const R wz = D == 3 ? w[2].N[c] : R(1);
        if (wz == R(0)) continue;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const R wxz = w[0].N[a] * wz;
            if (wxz == R(0)) continue;
            const R P0 = p[0] * wxz, P1 = p[1] * wxz, P2 = p[2] * wxz;
            Node8<R> *col = g.acc + (n0 + a * g.nny + c * plane);
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                const R wy = w[1].N[b];
                if (wy == R(0)) continue;
                red_add4(&col[b].a, R(0), P0 * wy, P1 * wy, P2 * wy);
            }
        }
    }
}

template <int D, typename R>
__global__ void __launch_bounds__(256, MPM_DMAP_MINB) k_dmap(PDev<D, R> P, GDev<R> g, StepParams sp) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= sp.np) return;
    AxisW<R> w[3];
    R p[3];
    dmap_core<D, R>(P, g, sp, i, w, p);
    dm2_scatter<D, R>(g, w, p);
}

// The same pass with the re-scatter of chained lanes merged (FP32 and FP64).
template <int D, typename R = float, bool GEN = true>
__global__ void __launch_bounds__(256, sizeof(R) == 8 ? MPM_CHAIN_MINB_F64 : MPM_DMAP_CHAIN_MINB) k_dmap_chain(PDev<D, R> P, GDev<R> g, StepParams sp) {
    // the particles in reverse block order: the pass before this one (the
    // fused pass) ends on the last particles and the one after it starts on
    // the first, so each pass starts on the data the previous one touched last
    // (still in L2; the column's double mapping touches ~130 MB, about L2's size)
    const int64_t i = (int64_t)(gridDim.x - 1 - blockIdx.x) * blockDim.x + threadIdx.x;
    const bool live = i < sp.np;
    AxisW<R> w[3];
    R p[3] = {0, 0, 0};
    int n0 = 0, key = dead_key();
    if (live) {
        dmap_core<D, R, GEN>(P, g, sp, i, w, p);
        n0 = key = window_n0<D, R>(g, w);
    } else {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            w[a].base = 0;
#pragma unroll
            for (int k = 0; k < 3; ++k) { w[a].N[k] = R(0.0); w[a].dN[k] = R(0.0); }
        }
    }
    dm2_scatter_chain<D, R>(g, w, n0, key, p);
}

// doublemapping3_OS!, utils_OS.jl:968-1016: grid velocity from the re-mapped
// momentum, BC, Δus = vs·ΔT (into the second half of the gather record).
// Clears mass and momentum for the next P2G.
template <int D, typename R>
__device__ __forceinline__ void dm3_node(const GDev<R> &g, const StepParams &sp, int i) {
    using T4 = typename Vec<R>::T4;
    const T4 a0 = g.acc[i].a;
    uint8_t bm = g.bcmask[i];
    if (a0.x == R(0) && a0.y == R(0) && a0.z == R(0) && a0.w == R(0) &&
        (g.bcval == nullptr || bm == 0)) {
        g.gat[i].b = mk4<R>(0, 0, 0, 0);
        return;
    }
    const R eps = (R)sp.meps;
    R md = a0.x < eps ? R(0) : R(1) / a0.x;
    R p[3] = {a0.y, a0.z, a0.w};
    R bv[3] = {R(0), R(0), R(0)};
    if (g.bcval) { T4 b = g.bcval[i]; bv[0] = b.x; bv[1] = b.y; bv[2] = b.z; }
    const R dt = (R)sp.dt;
    R du[3] = {0, 0, 0};
#pragma unroll
    for (int d = 0; d < D; ++d) {
        R vs = p[d] * md;
        if (bm & (1 << d)) vs = bv[d];
        du[d] = vs * dt;
    }
    g.gat[i].b = mk4<R>(du[0], du[1], du[2], 0);
    g.acc[i].a = mk4<R>(0, 0, 0, 0);
}

// Clears each processed block's flag (re-armed by the next scatter); the list
// count is reset by the host right after this launch.
template <int D, typename R>
__global__ void __launch_bounds__(128) k_dm3(GDev<R> g, StepParams sp) {
    const uint32_t n = *g.bcount;
    for (uint32_t k = blockIdx.x; k < n; k += gridDim.x) {
        const int b = (int)g.blist[k];
        const int i = block_node<D, R>(g, b, threadIdx.x);
        if (i >= 0) dm3_node<D, R>(g, sp, i);
        if (threadIdx.x == 0) g.bflag[b] = 0u;
    }
}

// Does the Drucker-Prager return change this trial stress (the shear or
// tension branch of dpP!, druckerprager.jl:89-155)?
// Particle fields staged in shared memory (slot-major, 256 threads per slot)
// by 4-byte cp.async at the start of the FP32 particle pass, so that their
// DRAM latency overlaps the node gathers instead of following them.
constexpr int PF_SIG = 0, PF_F = 6, PF_EPS = 15, PF_EPSQ = 21, PF_EPSK = 22, PF_VOL0 = 23, PF_M = 24,
              PF_V = 25, PF_MAT = 28, PF_COH = 29, PF_N = 30, PF_T = 256;

template <typename R> __device__ __forceinline__ R pf(const float *pre, int slot, const R *g) {
    return pre ? (R)pre[slot * PF_T] : ldcs(g);
}
__device__ __forceinline__ uint32_t pfu(const float *pre, int slot, const uint32_t *g) {
    return pre ? __float_as_uint(pre[slot * PF_T]) : ldcs(g);
}
__device__ __forceinline__ void cp_async4(float *dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
                 "l"(src)
                 : "memory");
}

// issue the copies of particle i's fields into this thread's slots
template <int D, typename R>
__device__ __forceinline__ void prefetch_particle(float *pre, const PDev<D, R> &P, int64_t i) {
    constexpr int NV = PDev<D, R>::NV, NF = PDev<D, R>::NF;
#pragma unroll
    for (int k = 0; k < NV; ++k) cp_async4(pre + (PF_SIG + k) * PF_T, P.sig[k] + i);
#pragma unroll
    for (int k = 0; k < NF; ++k) cp_async4(pre + (PF_F + k) * PF_T, P.F[k] + i);
#pragma unroll
    for (int k = 0; k < NV; ++k) cp_async4(pre + (PF_EPS + k) * PF_T, P.eps[k] + i);
    cp_async4(pre + PF_EPSQ * PF_T, P.epsq + i);
    cp_async4(pre + PF_EPSK * PF_T, P.epsk + i);
    cp_async4(pre + PF_VOL0 * PF_T, P.vol0 + i);
    cp_async4(pre + PF_M * PF_T, P.m + i);
#pragma unroll
    for (int d = 0; d < D; ++d) cp_async4(pre + (PF_V + d) * PF_T, P.v[d] + i);
    cp_async4(pre + PF_MAT * PF_T, P.mat + i);
    if (P.coh) cp_async4(pre + PF_COH * PF_T, P.coh + i);
    asm volatile("cp.async.commit_group;" ::: "memory");
}
__device__ __forceinline__ void prefetch_wait() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// 0: elastic, 1: shear branch, 2: tension branch (3D)
template <typename R> __device__ __forceinline__ int dp_branch(const R *s, const Mat<R> &M) {
    const R sm = (s[0] + s[1] + s[2]) * R(0.333333);
    const R d0 = s[0] - sm, d1 = s[1] - sm, d2 = s[2] - sm;
    const R tau = sqrt(R(0.5) * (d0 * d0 + d1 * d1 + d2 * d2) + s[3] * s[3] + s[4] * s[4] + s[5] * s[5]);
    const R fs = tau + M.qphi * sm - M.kphi;
    const R BF = (tau - M.tb) - (M.ab * (sm - M.st));
    if ((sm < M.st) && (fs > R(0))) return 1;
    if (sm >= M.st) return BF > R(0) ? 1 : 2;
    return 0;
}
template <typename R> __device__ __forceinline__ bool dp_yielding(const R *s, const Mat<R> &M) {
    return dp_branch<R>(s, M) != 0;
}

__device__ __forceinline__ bool hash_keep(int64_t i, uint32_t salt, uint32_t every) {
    uint32_t x = (uint32_t)i * 0x9E3779B1u ^ salt;
    x ^= x >> 16; x *= 0x85EBCA6Bu; x ^= x >> 13; x *= 0xC2B2AE35u; x ^= x >> 16;
    return every <= 1 || x % every == 0;
}

// restated 3D Mohr-Coulomb parameters of a material
template <typename R> __device__ __forceinline__ mc3d::Par mc3d_par(const Mat<R> &M) {
    return mc3d::Par{(double)M.K, (double)M.G, (double)M.c, (double)M.phi, (double)M.psi,
                     (double)M.sigt, (double)M.sphi, (double)M.cphi, (double)M.tphi, (double)M.tpsi};
}

// one row of surrogate features (and, when `out` is given, its target; when
// `s0` is given -- a deferred Mohr-Coulomb return -- the rotated pre-increment
// stress, in the target row, which deferral leaves unused)
template <typename R>
__device__ __forceinline__ void surr_features(const SurrCtx &c, int64_t i, const R *trial, const R *de, R eq,
                                              const Mat<R> &M, const R *out, const R *s0 = nullptr,
                                              float tag = 0.0f) {
    const uint32_t r = atomicAdd(c.cnt, 1u);
    if (r >= c.cap) return;
    float4 *f = reinterpret_cast<float4 *>(c.feat + (size_t)r * 16);
    f[0] = make_float4((float)trial[0], (float)trial[1], (float)trial[2], (float)trial[3]);
    f[1] = make_float4((float)trial[4], (float)trial[5], (float)de[0], (float)de[1]);
    f[2] = make_float4((float)de[2], (float)de[3], (float)de[4], (float)de[5]);
    f[3] = make_float4((float)eq, (float)M.c, (float)M.phi, tag);   // tag: the network ignores column 15
    if (out) {
#pragma unroll
        for (int k = 0; k < 6; ++k) c.tgt[(size_t)r * 6 + k] = (float)out[k];
    }
    if (s0 && c.tgt) {
#pragma unroll
        for (int k = 0; k < 6; ++k) c.tgt[(size_t)r * 6 + k] = (float)s0[k];
    }
    if (c.list) c.list[r] = (uint32_t)i;
}

// Everything of G2P_OS! after the gathers, plus liE! and dpP!/mcP! and the
// DM1 position update: x (in/out, FP64), tT = ΣN·vsT, dF = ΣΔu⊗∇N.  Stores
// the particle and returns the new stress s and volume vol for the next P2G.
template <int D, typename R, bool MC3 = false>
__device__ __forceinline__ void update_particle(const PDev<D, R> &P, const GDev<R> &g, const StepParams &sp,
                                                int64_t i, double *x, const R *tT, const R *dF, R *s, R &vol,
                                                const float *pre = nullptr, double *Jout = nullptr,
                                                bool *deferred = nullptr) {
    constexpr int NV = PDev<D, R>::NV, NF = PDev<D, R>::NF;
    // position: ξ += ΔT·ΣN·vsT, accumulated in FP64
#pragma unroll
    for (int d = 0; d < D; ++d) x[d] += (double)tT[d] * sp.dt;
    const R dT1 = R(1) / (R)sp.dt;
    R de[6], ev;
    if (D == 2) {
        R exx = dF[0] * dT1, eyy = dF[3] * dT1, exy = R(0.5) * (dF[1] + dF[2]) * dT1;
        ev = sqrt(exx * exx + eyy * eyy + R(2) * exy * exy);
        de[0] = dF[0]; de[1] = dF[3]; de[2] = R(0); de[3] = dF[1] + dF[2];
    } else {
        R exx = dF[0] * dT1, eyy = dF[4] * dT1, ezz = dF[8] * dT1;
        R exy = R(0.5) * (dF[1] + dF[3]) * dT1, eyz = R(0.5) * (dF[5] + dF[7]) * dT1,
          exz = R(0.5) * (dF[2] + dF[6]) * dT1;
        ev = sqrt(exx * exx + eyy * eyy + ezz * ezz + R(2) * (exy * exy + eyz * eyz + exz * exz));
        de[0] = dF[0]; de[1] = dF[4]; de[2] = dF[8];
        de[3] = dF[1] + dF[3]; de[4] = dF[5] + dF[7]; de[5] = dF[2] + dF[6];
    }
    // strain
    if (D == 2) {
        stcs(P.eps[0] + i, pf(pre, PF_EPS + 0, P.eps[0] + i) + de[0]);
        stcs(P.eps[1] + i, pf(pre, PF_EPS + 1, P.eps[1] + i) + de[1]);
        stcs(P.eps[3] + i, pf(pre, PF_EPS + 3, P.eps[3] + i) + de[3]);
    } else {
#pragma unroll
        for (int k = 0; k < 6; ++k) stcs(P.eps[k] + i, pf(pre, PF_EPS + k, P.eps[k] + i) + de[k]);
    }
    stcs(P.epsv + i, ev);
    // F <- (I + ΔF) F, formed as F + ΔF·F; J = det F in FP64; Ω = J Ω0.
    // In FP32, (1 + ΔF_ii) would keep ΔF_ii (≈1e-5 per step) only to the
    // absolute 6e-8 of 1's half-ulp -- a relative error up to ~1e-2 that repeats
    // with the same sign while a column settles under gravity and biases J,
    // hence the volumes and the nodal forces.  F + ΔF·F rounds once, at F's
    // own half-ulp, where the rounding changes sign from step to step.
    R f[9], fn[9];
#pragma unroll
    for (int k = 0; k < NF; ++k) f[k] = pf(pre, PF_F + k, P.F[k] + i);
    double J;
    if (D == 2) {
        fn[0] = f[0] + (dF[0] * f[0] + dF[1] * f[2]);
        fn[1] = f[1] + (dF[0] * f[1] + dF[1] * f[3]);
        fn[2] = f[2] + (dF[3] * f[2] + dF[2] * f[0]);
        fn[3] = f[3] + (dF[3] * f[3] + dF[2] * f[1]);
        J = (double)fn[0] * (double)fn[3] - (double)fn[1] * (double)fn[2];
    } else {
        fn[0] = f[0] + (dF[0] * f[0] + dF[1] * f[3] + dF[2] * f[6]);
        fn[1] = f[1] + (dF[0] * f[1] + dF[1] * f[4] + dF[2] * f[7]);
        fn[2] = f[2] + (dF[0] * f[2] + dF[1] * f[5] + dF[2] * f[8]);
        fn[3] = f[3] + (dF[4] * f[3] + dF[3] * f[0] + dF[5] * f[6]);
        fn[4] = f[4] + (dF[4] * f[4] + dF[3] * f[1] + dF[5] * f[7]);
        fn[5] = f[5] + (dF[4] * f[5] + dF[3] * f[2] + dF[5] * f[8]);
        fn[6] = f[6] + (dF[8] * f[6] + dF[7] * f[3] + dF[6] * f[0]);
        fn[7] = f[7] + (dF[8] * f[7] + dF[7] * f[4] + dF[6] * f[1]);
        fn[8] = f[8] + (dF[8] * f[8] + dF[7] * f[5] + dF[6] * f[2]);
        double g0 = fn[0], g1 = fn[1], g2 = fn[2], g3 = fn[3], g4 = fn[4], g5 = fn[5], g6 = fn[6],
               g7 = fn[7], g8 = fn[8];
        J = g0 * g4 * g8 + g1 * g5 * g6 + g2 * g3 * g7 - g6 * g4 * g2 - g7 * g5 * g0 - g8 * g3 * g1;
    }
#pragma unroll
    for (int k = 0; k < NF; ++k) stcs(P.F[k] + i, fn[k]);
    vol = (R)(J * (double)pf(pre, PF_VOL0, P.vol0 + i));
    stcs(P.vol + i, vol);
    if (Jout) *Jout = J;
    // stress: liE! then dpP! / mcP! (OS_MUSL.jl:82-96)
    Mat<R> M = g.mat[pfu(pre, PF_MAT, P.mat + i)];
    if (P.coh) {
        // one material per particle differing only in cohesion (a random
        // field): the cohesion-dependent constants of druckerprager.jl:39-44
        const R c = pf(pre, PF_COH, P.coh + i);
        M.c = c;
        M.kphi = c * M.kc;
        M.st = fmin(M.sigt, M.kphi / M.qphi);
        M.tb = M.kphi - M.qphi * M.st;
    }
    R srot[6];
#pragma unroll
    for (int k = 0; k < NV; ++k) s[k] = pf(pre, PF_SIG + k, P.sig[k] + i);
    lin_elastic<D, R>(s, dF, de, M, srot);
    if (sp.plastic && (sp.constitutive == 1 || (sp.constitutive == 2 && D == 2))) {
        R eq = pf(pre, PF_EPSQ, P.epsq + i), ek = pf(pre, PF_EPSK, P.epsk + i);
        if (D == 3 && sp.constitutive == 1 && sp.surr.mode == 2) {
            if (dp_yielding<R>(s, M)) {
                surr_features<R>(sp.surr, i, s, de, eq, M, nullptr);
                if (deferred) *deferred = true;
            }
        } else if (D == 3 && sp.constitutive == 1 && sp.surr.mode == 1) {
            R trial[6];
#pragma unroll
            for (int k = 0; k < 6; ++k) trial[k] = s[k];
            const R eq0 = eq;
            drucker_prager<D, R>(s, eq, ek, M);
            if (eq != eq0 && hash_keep(i, sp.surr.salt, sp.surr.every)) surr_features<R>(sp.surr, i, trial, de, eq0, M, s);
        } else if (sp.constitutive == 1) {
            drucker_prager<D, R>(s, eq, ek, M);
        } else {
            mohr_coulomb_2d<R>(s, eq, ek, M);
        }
        stcs(P.epsq + i, eq);
        stcs(P.epsk + i, ek);
    } else if (MC3 && D == 3 && sp.plastic && sp.constitutive == 2) {
        // restated 3D Mohr-Coulomb, FP64 (mohrcoulomb.jl:152-455, commented out there)
        double sd[6], s0d[6], ded[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) { sd[k] = s[k]; s0d[k] = srot[k]; ded[k] = de[k]; }
        const mc3d::Par mp = mc3d_par<R>(M);
        if (mc3d::surely_elastic(sd, mp)) {
            // elastic by a margin above the FP32 screen's error: the FP64
            // classification would say ELASTIC, the stress stays the trial one
        } else if (sp.surr.mode == 2) {
            // surrogate: a yielding trial keeps its trial stress and is queued
            // (features, and the rotated pre-increment stress the fallback needs)
            mc3d::Inv v;
            double ft, fs;
            mc3d::invariants(sd, v);
            const int mode = mc3d::yield(v, mp, ft, fs);
            if (mode != mc3d::ELASTIC) {
                const R eq = pf(pre, PF_EPSQ, P.epsq + i);
                surr_features<R>(sp.surr, i, s, de, eq, M, nullptr, srot, (float)mode);
                if (deferred) *deferred = true;
            }
        } else {
            const mc3d::Ret r = mc3d::mohr_coulomb_3d(sd, s0d, ded, mp);
            if (r.yielded) {
                R trial[6];
#pragma unroll
                for (int k = 0; k < 6; ++k) { trial[k] = s[k]; s[k] = (R)sd[k]; }
                const R eq0 = pf(pre, PF_EPSQ, P.epsq + i);
                stcs(P.epsq + i, (R)((double)eq0 + r.dq));
                if (sp.surr.mode == 1 && hash_keep(i, sp.surr.salt, sp.surr.every))
                    surr_features<R>(sp.surr, i, trial, de, eq0, M, s);
            }
        }
    }
#pragma unroll
    for (int k = 0; k < NV; ++k) stcs(P.sig[k] + i, s[k]);
#pragma unroll
    for (int d = 0; d < D; ++d) stcs(P.x[d] + i, x[d]);
    bool bad = !(J > 0.0);
    bool nan = !isfinite(x[0]) || !isfinite(x[1]) || !isfinite((double)s[0]) || !isfinite((double)s[1]);
    if (bad) atomicOr(g.err, ERR_J);
    if (nan) atomicOr(g.err, ERR_NAN);
}

// The per-particle body of the G2P pass: gathers, DM1 velocity (USL), the
// update (update_particle) and, without FUSE, the MVL cell sums.  Returns the
// updated position x, stress s and volume vol for the next scatter.
template <int D, typename R, bool FUSE, bool MC3, bool USL>
__device__ __forceinline__ void g2p_core(const PDev<D, R> &P, const GDev<R> &g, const StepParams &sp, int64_t i,
                                         float *pre, double *x, AxisW<R> *w, R *s, R &vol,
                                         bool *deferred = nullptr) {
    load_x<D, R>(P, i, x);
    particle_weights<D, R>(x, g, w);
    const int n0 = window_n0<D, R>(g, w);
    const int plane = g.nnx * g.nny;
    R tT[3] = {0, 0, 0};
    R dF[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    constexpr int NC = D == 3 ? 3 : 1;
    // ΣΔu⊗∇N = Σ(Δu - Δu_c)⊗∇N since Σ∇N = 0 (uGIMP partition of unity); the
    // window-centre node's Δu_c is subtracted before the products, which keeps
    // the FP32 sum from cancelling when the motion is mostly a translation.
    // Separable sums: per (x, z) column, A = ΣNy·Δu', B = ΣdNy·Δu', T = ΣNy·vsT;
    // then ∂/∂x += dNx·Nz·A, ∂/∂y += Nx·Nz·B, ∂/∂z += Nx·dNz·A, tT += Nx·Nz·T.
    // USL: Δu = vsT·dt (OS_USL.jl), taken from the first half of the record and
    // scaled after the sums; the DM1 velocity update gathers as / vs alongside.
    const int ncen = n0 + g.nny + 1 + (D == 3 ? plane : 0);
    const auto duc = USL ? g.gat[ncen].a : g.gat[ncen].b;
    R ta[3] = {0, 0, 0}, tv[3] = {0, 0, 0};
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        const R wz = D == 3 ? w[2].N[c] : R(1);
        const R gz = D == 3 ? w[2].dN[c] : R(0);
        if (wz == R(0)) continue;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const R wx = w[0].N[a];
            if (wx == R(0)) continue;
            const int col = n0 + a * g.nny + c * plane;
            R T[3] = {0, 0, 0}, A[3] = {0, 0, 0}, B[3] = {0, 0, 0}, Sa[3] = {0, 0, 0}, Sv[3] = {0, 0, 0};
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                const R wy = w[1].N[b], gy = w[1].dN[b];
                // a node of zero weight (it then has zero dN too) is not read,
                // and its sums are formed with Δu = Δu_c and q = 0, i.e. add
                // nothing: the load is skipped by a predicate, the sums run
                // unconditionally (no divergent branch in the inner loop)
                Node8<R> q;
                q.a = mk4<R>(0, 0, 0, 0);
                q.b = q.a;
                if (wy != R(0)) q = g.gat[col + b];
                const auto du = USL ? q.a : (wy != R(0) ? q.b : duc);
                if constexpr (std::is_same<R, float>::value) {
                    // x and y components as packed FP32 pairs
                    const float2 w2 = make_float2(wy, wy), g2 = make_float2(gy, gy);
                    const float2 u01 = __fadd2_rn(make_float2(du.x, du.y), make_float2(-duc.x, -duc.y));
                    const float2 t01 = __ffma2_rn(w2, make_float2(q.a.x, q.a.y), make_float2(T[0], T[1]));
                    const float2 a01 = __ffma2_rn(w2, u01, make_float2(A[0], A[1]));
                    const float2 b01 = __ffma2_rn(g2, u01, make_float2(B[0], B[1]));
                    T[0] = t01.x; T[1] = t01.y; T[2] += wy * q.a.z;
                    A[0] = a01.x; A[1] = a01.y; B[0] = b01.x; B[1] = b01.y;
                    if (D == 3) {
                        const float u2 = du.z - duc.z;
                        A[2] += wy * u2; B[2] += gy * u2;
                    }
                } else {
                    const R u[3] = {du.x - duc.x, du.y - duc.y, du.z - duc.z};
                    T[0] += wy * q.a.x; T[1] += wy * q.a.y; T[2] += wy * q.a.z;
#pragma unroll
                    for (int k = 0; k < D; ++k) { A[k] += wy * u[k]; B[k] += gy * u[k]; }
                }
                if (USL) {
                    Sa[0] += wy * q.b.x; Sa[1] += wy * q.b.y; Sa[2] += wy * q.b.z;
                    if (sp.need_vs) {
                        const auto vv = g.gvs[col + b];
                        Sv[0] += wy * vv.x; Sv[1] += wy * vv.y; Sv[2] += wy * vv.z;
                    }
                }
            }
            const R wxz = wx * wz, gxz = w[0].dN[a] * wz;
#pragma unroll
            for (int k = 0; k < D; ++k) tT[k] += wxz * T[k];
            if (USL) {
#pragma unroll
                for (int k = 0; k < D; ++k) { ta[k] += wxz * Sa[k]; tv[k] += wxz * Sv[k]; }
            }
            if (D == 2) {
                dF[0] += gxz * A[0]; dF[1] += wxz * B[0];
                dF[2] += gxz * A[1]; dF[3] += wxz * B[1];
            } else {
                const R xdz = wx * gz;
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    dF[3 * k + 0] += gxz * A[k];
                    dF[3 * k + 1] += wxz * B[k];
                    dF[3 * k + 2] += xdz * A[k];
                }
            }
        }
    }
    if (USL) {
        // Δu = vsT·dt
        const R dt = (R)sp.dt;
#pragma unroll
        for (int k = 0; k < D * D; ++k) dF[k] *= dt;
        // doublemapping1_a_USL_OS! / doublemapping1_OS! (OS_USL.jl:185-320)
        const R FLIP = (R)sp.FLIP, PIC = (R)sp.PIC;
        if (pre) prefetch_wait();
#pragma unroll
        for (int d = 0; d < D; ++d) {
            const R vo = pf(pre, PF_V + d, P.v[d] + i);
            const R vn = sp.va == 0 ? FLIP * vo + PIC * tT[d] + ta[d] * dt : FLIP * (vo + (tT[d] - tv[d])) + PIC * tT[d];
            stcs(P.v[d] + i, vn);
            if (pre) pre[(PF_V + d) * PF_T] = (float)vn;
        }
    }
    int cell = 0;
    if (!FUSE && sp.mvl) {
        // vollock1_OS!: the cell of the step's start (the reference's p2c)
        int ci[3];
        particle_cell<D, R>(x, g, ci);
        const int cx = clampi(ci[0], 0, g.ax[0].nc - 1), cy = clampi(ci[1], 0, g.ax[1].nc - 1);
        const int cz = D == 3 ? clampi(ci[2], 0, g.ax[2].nc - 1) : 0;
        cell = (cz * g.ax[0].nc + cx) * g.ax[1].nc + cy;
    }
    if (pre) prefetch_wait();
    update_particle<D, R, MC3>(P, g, sp, i, x, tT, dF, s, vol, pre, nullptr, deferred);
    if (!FUSE && sp.mvl) {
        const R sm = (s[0] + s[1] + s[2]) * R(0.333333);
        atomicAdd(&g.csigm[cell], vol * sm);
        atomicAdd(&g.comega[cell], vol);
        g.pcell[i] = (uint32_t)cell;
    }
}

// ---------------------------------------------------------------------------
// G2P_OS! (utils_OS.jl:1025-1153) + the position update of DM1 + liE! +
// dpP!/mcP!.  With FUSE, the next step's P2G scatters the updated particle
// (resetmpstatus_OS! + P2G_OS! at the new position, gravity sp.G).
// ---------------------------------------------------------------------------
template <int D, typename R, bool FUSE, bool MC3 = false, bool USL = false>
__global__ void __launch_bounds__(256, MPM_P_MINB) k_g2p(PDev<D, R> P, GDev<R> g, StepParams sp) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= sp.np) return;
    extern __shared__ float g2p_pre[];   // PF_N slots x 256 threads when sp.prefetch
    float *pre = nullptr;
    if (sizeof(R) == 4 && sp.prefetch) {
        pre = g2p_pre + threadIdx.x;
        prefetch_particle<D, R>(pre, P, i);
    }
    double x[3];
    AxisW<R> w[3];
    R s[6], vol;
    g2p_core<D, R, FUSE, MC3, USL>(P, g, sp, i, pre, x, w, s, vol);
    if (FUSE) {
        if (!particle_weights<D, R>(x, g, w)) { atomicOr(g.err, ERR_OOG); return; }
        R v[3];
#pragma unroll
        for (int d = 0; d < D; ++d) v[d] = pf(pre, PF_V + d, P.v[d] + i);
        if (D == 2) v[2] = R(0);
        p2g_scatter<D, R>(g, w, pf(pre, PF_M, P.m + i), vol, v, s, (R)sp.G);
    }
}

// The same pass (FUSE) with the scatter of chained lanes merged (FP32 and FP64).
// MINB: resident CTAs per SM in FP32 (the register cap); 4 by default, 3 for
// particle-pass variant 3 (models whose fused pass runs faster with 85
// registers and fewer warps, e.g. the random-field slope).
template <int D, bool MC3 = false, bool USL = false, typename R = float, int MINB = MPM_P_MINB>
__global__ void __launch_bounds__(256, sizeof(R) == 8 ? MPM_CHAIN_MINB_F64 : MINB) k_g2p_chain(PDev<D, R> P, GDev<R> g, StepParams sp) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    bool live = i < sp.np;
    double x[3];
    AxisW<R> w[3];
    R s[6] = {0, 0, 0, 0, 0, 0}, vol = 0, v[3] = {0, 0, 0}, m = 0;
    // FP32: the particle's fields are requested (cp.async into shared memory)
    // before the gathers, so their DRAM latency overlaps the node reads
    extern __shared__ float g2p_pre[];   // PF_N slots x 256 threads when sp.prefetch
    float *pre = nullptr;
    if (sizeof(R) == 4 && sp.prefetch && live) {
        pre = g2p_pre + threadIdx.x;
        prefetch_particle<D, R>(pre, P, i);
    }
    if (live) {
        bool deferred = false;   // (surrogate) return queued: scattered after the accept-or-fallback pass
        g2p_core<D, R, true, MC3, USL>(P, g, sp, i, pre, x, w, s, vol, &deferred);
        if (deferred) {
            live = false;
        } else if (!particle_weights<D, R>(x, g, w)) {
            atomicOr(g.err, ERR_OOG);
            live = false;
        } else {
#pragma unroll
            for (int d = 0; d < D; ++d) v[d] = pf(pre, PF_V + d, P.v[d] + i);
            m = pf(pre, PF_M, P.m + i);
        }
    }
    int n0 = 0, key = dead_key();
    if (live) {
        n0 = key = window_n0<D, R>(g, w);
    } else {
        m = R(0.0);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            w[a].base = 0;
#pragma unroll
            for (int k = 0; k < 3; ++k) { w[a].N[k] = R(0.0); w[a].dN[k] = R(0.0); }
        }
    }
    MarkState mk;
    if (live) mk = mark_begin<D, R>(g, w);
    p2g_scatter_chain<D, R>(g, w, n0, key, m, vol, v, s, (R)sp.G);
    if (live) mark_end<R>(g, mk);
}

// vollock2_OS! + the next step's P2G: the particle's mean stress is replaced by
// the volume-weighted mean of its start-of-step cell (utils_OS.jl:1162-1257),
// then it scatters at its new position.
template <int D, typename R>
__global__ void __launch_bounds__(256) k_mvl_p2g(PDev<D, R> P, GDev<R> g, StepParams sp) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= sp.np) return;
    constexpr int NV = PDev<D, R>::NV;
    const uint32_t c = g.pcell[i];
    const R cm = g.csigm[c] / g.comega[c];
    R s[6];
#pragma unroll
    for (int k = 0; k < NV; ++k) s[k] = P.sig[k][i];
    const R sm = (s[0] + s[1] + s[2]) * R(0.333333);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        s[k] = (s[k] - sm) + cm;
        P.sig[k][i] = s[k];
    }
    double x[3];
    load_x<D, R>(P, i, x);
    AxisW<R> w[3];
    if (!particle_weights<D, R>(x, g, w)) { atomicOr(g.err, ERR_OOG); return; }
    R v[3] = {P.v[0][i], P.v[1][i], D == 3 ? P.v[2][i] : R(0)};
    p2g_scatter<D, R>(g, w, P.m[i], P.vol[i], v, s, (R)sp.G);
}

// The same pass with the scatters of chained lanes merged (p2g_scatter_chain).
template <int D, typename R = float>
__global__ void __launch_bounds__(256) k_mvl_p2g_chain(PDev<D, R> P, GDev<R> g, StepParams sp) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    bool live = i < sp.np;
    constexpr int NV = PDev<D, R>::NV;
    R s[6] = {0, 0, 0, 0, 0, 0}, v[3] = {0, 0, 0}, m = R(0.0), vol = R(0.0);
    AxisW<R> w[3];
    if (live) {
        const uint32_t c = g.pcell[i];
        const R cm = g.csigm[c] / g.comega[c];
#pragma unroll
        for (int k = 0; k < NV; ++k) s[k] = P.sig[k][i];
        const R sm = (s[0] + s[1] + s[2]) * R(0.333333);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            s[k] = (s[k] - sm) + cm;
            P.sig[k][i] = s[k];
        }
        double x[3];
        load_x<D, R>(P, i, x);
        if (!particle_weights<D, R>(x, g, w)) {
            atomicOr(g.err, ERR_OOG);
            live = false;
        } else {
            v[0] = P.v[0][i]; v[1] = P.v[1][i];
            if (D == 3) v[2] = P.v[2][i];
            m = P.m[i];
            vol = P.vol[i];
        }
    }
    int n0 = 0, key = dead_key();
    if (live) {
        n0 = key = window_n0<D, R>(g, w);
    } else {
        m = vol = R(0.0);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            w[a].base = 0;
#pragma unroll
            for (int k = 0; k < 3; ++k) { w[a].N[k] = R(0.0); w[a].dN[k] = R(0.0); }
        }
    }
    MarkState mk;
    if (live) mk = mark_begin<D, R>(g, w);
    p2g_scatter_chain<D, R>(g, w, n0, key, m, vol, v, s, (R)sp.G);
    if (live) mark_end<R>(g, mk);
}

// Finish the deferred returns: accept the surrogate's stress when its yield
// residual |f(s_hat)| / max(kphi, |qphi s_hat_m|, s_ref) is within tol (f of the
// branch the trial stress takes: the shear cone, or the tension cut-off
// s_m = st), else fall back to the plain return.  The plastic strains follow
// the plain return's closed-form multiplier either way.  stats[0] += rows,
// stats[1] += fallbacks.
template <typename R>
__global__ void __launch_bounds__(256) k_surr_fix(PDev<3, R> P, GDev<R> g, SurrCtx c, const float *out, float tol,
                                                  float sref, unsigned long long *stats) {
    const uint32_t n = min(*c.cnt, c.cap);
    uint32_t nfall = 0, nrows = 0;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int64_t i = c.list[k];
        Mat<R> M = g.mat[P.mat[i]];
        if (P.coh) {
            const R cc = P.coh[i];
            M.c = cc;
            M.kphi = cc * M.kc;
            M.st = fmin(M.sigt, M.kphi / M.qphi);
            M.tb = M.kphi - M.qphi * M.st;
        }
        R sp[6], sh[6];
#pragma unroll
        for (int q = 0; q < 6; ++q) { sp[q] = P.sig[q][i]; sh[q] = (R)out[(size_t)k * 6 + q]; }
        R eq = P.epsq[i], ek = P.epsk[i];
        const bool tension = dp_branch<R>(sp, M) == 2;
        drucker_prager<3, R>(sp, eq, ek, M);   // the plain return: fallback and plastic strains
        const R hm = (sh[0] + sh[1] + sh[2]) * R(0.333333);
        const R d0 = sh[0] - hm, d1 = sh[1] - hm, d2 = sh[2] - hm;
        const R htau = sqrt(R(0.5) * (d0 * d0 + d1 * d1 + d2 * d2) + sh[3] * sh[3] + sh[4] * sh[4] + sh[5] * sh[5]);
        const R scale = fmax(fmax(M.kphi, fabs(M.qphi * hm)), (R)sref);
        const R resid = tension ? fabs(hm - M.st) : fabs(htau + M.qphi * hm - M.kphi);
        const bool ok = isfinite((double)resid) && resid <= (R)tol * scale;
#pragma unroll
        for (int q = 0; q < 6; ++q) P.sig[q][i] = ok ? sh[q] : sp[q];
        P.epsq[i] = eq;
        P.epsk[i] = ek;
        nfall += ok ? 0u : 1u;
        nrows += 1u;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        nfall += __shfl_xor_sync(0xffffffffu, nfall, o);
        nrows += __shfl_xor_sync(0xffffffffu, nrows, o);
    }
    if ((threadIdx.x & 31) == 0 && nrows) {
        atomicAdd(&stats[0], (unsigned long long)nrows);
        atomicAdd(&stats[1], (unsigned long long)nfall);
    }
}

// The deferred restated 3D Mohr-Coulomb returns (mohr_coulomb_3d): keep the
// network's stress σ̂ when it lies on the yield surface the trial crossed (its
// mode, tensile or shear, is tagged in feature column 15 at deferral) --
// |f_mode(σ̂)| <= tol·scale and neither yield function above tol·scale, with
// scale = max(c, |σ̂m|·tanφ, sref) -- else run the plain return from the
// trial stress (stored as the particle's stress), the rotated pre-increment
// stress (kept in the row's target slot) and the strain increment (features
// 6..11); the acceptance test evaluates the yield functions in FP32.  An
// accepted row's ϵq grows by √(2/3)·|e|, e = dev(σtrial - σ̂)/(2G),
// the plastic shear strain of the correction (ϵq does not enter the restated
// return: it has no softening).
template <typename R>
__global__ void __launch_bounds__(256) k_surr_fix_mc(PDev<3, R> P, GDev<R> g, SurrCtx c, const float *out, float tol,
                                                     float sref, unsigned long long *stats) {
    const uint32_t n = min(*c.cnt, c.cap);
    uint32_t nfall = 0, nrows = 0;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int64_t i = c.list[k];
        Mat<R> M = g.mat[P.mat[i]];
        if (P.coh) M.c = P.coh[i];
        const mc3d::Par mp = mc3d_par<R>(M);
        double tr[6], sh[6];
        float shf[6];
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            tr[q] = (double)P.sig[q][i];
            shf[q] = out[(size_t)k * 6 + q];
            sh[q] = (double)shf[q];
        }
        // the acceptance test in FP32 (the plain return stays FP64)
        float fth, fsh, smh;
        mc3d::yield_f32(shf, mp, fth, fsh, smh);
        const int type = (int)c.feat[(size_t)k * 16 + 15];   // the trial's mode, tagged at deferral
        const float scale = fmaxf(fmaxf((float)mp.c, fabsf(smh) * (float)mp.tphi), sref);
        const float fact = type == mc3d::TENSILE ? fth : fsh;
        const bool ok = isfinite(fact) && isfinite(fsh) && isfinite(fth) && fabsf(fact) <= tol * scale &&
                        fmaxf(fth, fsh) <= tol * scale;
        double dq;
        if (ok) {
            const double ds = ((tr[0] - sh[0]) + (tr[1] - sh[1]) + (tr[2] - sh[2])) / 3.0;
            double ee = 0.0;
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                const double e = ((tr[q] - sh[q]) - ds) / (2.0 * mp.G);
                ee += e * e;
            }
#pragma unroll
            for (int q = 3; q < 6; ++q) {
                const double e = (tr[q] - sh[q]) / (2.0 * mp.G);
                ee += 2.0 * e * e;
            }
            dq = sqrt(2.0 / 3.0 * ee);
        } else {
            double s0[6], de[6];
#pragma unroll
            for (int q = 0; q < 6; ++q) {
                s0[q] = (double)c.tgt[(size_t)k * 6 + q];
                de[q] = (double)c.feat[(size_t)k * 16 + 6 + q];
            }
            const mc3d::Ret r = mc3d::mohr_coulomb_3d(tr, s0, de, mp);
            dq = r.dq;
        }
#pragma unroll
        for (int q = 0; q < 6; ++q) P.sig[q][i] = (R)(ok ? sh[q] : tr[q]);
        P.epsq[i] = (R)((double)P.epsq[i] + dq);
        nfall += ok ? 0u : 1u;
        nrows += 1u;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        nfall += __shfl_xor_sync(0xffffffffu, nfall, o);
        nrows += __shfl_xor_sync(0xffffffffu, nrows, o);
    }
    if ((threadIdx.x & 31) == 0 && nrows) {
        atomicAdd(&stats[0], (unsigned long long)nrows);
        atomicAdd(&stats[1], (unsigned long long)nfall);
    }
}

// P2G_OS! of the particles whose returns the surrogate pass finished (the rows
// of the deferred list); the fused pass scattered all the others.
template <int D, typename R>
__global__ void __launch_bounds__(256) k_p2g_list(PDev<D, R> P, GDev<R> g, StepParams sp, const uint32_t *list,
                                                  const uint32_t *cnt, uint32_t cap) {
    const uint32_t n = min(*cnt, cap);
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int64_t i = list[k];
        double x[3];
        load_x<D, R>(P, i, x);
        AxisW<R> w[3];
        if (!particle_weights<D, R>(x, g, w)) { atomicOr(g.err, ERR_OOG); continue; }
        R v[3] = {P.v[0][i], P.v[1][i], D == 3 ? P.v[2][i] : R(0)};
        R s[6];
#pragma unroll
        for (int q = 0; q < PDev<D, R>::NV; ++q) s[q] = P.sig[q][i];
        p2g_scatter<D, R>(g, w, P.m[i], P.vol[i], v, s, (R)sp.G);
    }
}

// P2G_OS! alone (the scatter after the surrogate's accept-or-fallback pass),
// with the scatters of chained lanes merged.
template <int D, typename R = float>
__global__ void __launch_bounds__(256, sizeof(R) == 8 ? MPM_CHAIN_MINB_F64 : MPM_P_MINB)
    k_p2g_chain(PDev<D, R> P, GDev<R> g, StepParams sp) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    bool live = i < sp.np;
    AxisW<R> w[3];
    R s[6] = {0, 0, 0, 0, 0, 0}, vol = 0, v[3] = {0, 0, 0}, m = 0;
    if (live) {
        double x[3];
        load_x<D, R>(P, i, x);
        if (!particle_weights<D, R>(x, g, w)) {
            atomicOr(g.err, ERR_OOG);
            live = false;
        } else {
#pragma unroll
            for (int d = 0; d < D; ++d) v[d] = ldcs(P.v[d] + i);
#pragma unroll
            for (int k = 0; k < PDev<D, R>::NV; ++k) s[k] = ldcs(P.sig[k] + i);
            m = ldcs(P.m + i);
            vol = ldcs(P.vol + i);
        }
    }
    int n0 = 0, key = dead_key();
    if (live) {
        n0 = key = window_n0<D, R>(g, w);
    } else {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            w[a].base = 0;
#pragma unroll
            for (int k = 0; k < 3; ++k) { w[a].N[k] = R(0.0); w[a].dN[k] = R(0.0); }
        }
    }
    MarkState mk;
    if (live) mk = mark_begin<D, R>(g, w);
    p2g_scatter_chain<D, R>(g, w, n0, key, m, vol, v, s, (R)sp.G);
    if (live) mark_end<R>(g, mk);
}

// p2c of the current positions, 1-based, in the original particle order.
template <int D, typename R>
__global__ void k_p2c(PDev<D, R> P, GDev<R> g, int64_t np, int64_t *out) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    double xp[3];
    load_x<D, R>(P, i, xp);
    // p2c = cld(y - y1, dy) + fld(z - z1, dz)*ncy*ncx + fld(x - x1, dx)*ncy
    double cy = jl_cld(xp[1] - g.ax[1].x1, g.ax[1].h);
    double cx = jl_fld(xp[0] - g.ax[0].x1, g.ax[0].h);
    double v;
    if (D == 2) v = cy + cx * (double)g.ax[1].nc;
    else {
        double cz = jl_fld(xp[2] - g.ax[2].x1, g.ax[2].h);
        v = cy + cz * (double)g.ax[1].nc * (double)g.ax[0].nc + cx * (double)g.ax[1].nc;
    }
    int64_t r = (v >= -9.0e18 && v <= 9.0e18) ? (int64_t)trunc(v) : (int64_t)(-1);
    out[P.orig[i]] = r;
}

}  // namespace mpm
