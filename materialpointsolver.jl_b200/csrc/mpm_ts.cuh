// mpm_ts.cuh -- two-phase (coupling = :TS) MUSL step: procedure!(…, Val(:TS),
// Val(:MUSL)), src/solvers/TS_MUSL.jl:13-54, kernels of src/solvers/utils_TS.jl.
//
// The reference's two-phase path does not run as shipped; this restatement
// keeps its arithmetic and repairs three defects:
//   * submit_work! calls workflow(…, Val(coupling), Val(scheme), Val(va))
//     (src/solver.jl:84-85) while the :TS procedure! takes two Val arguments
//     (TS_MUSL.jl:13-23): the step runs whatever va is;
//   * G2P_TS! reads mp.ρs_init / mp.ρw_init (utils_TS.jl:849-850, 953-954),
//     fields Particle2D/3D do not have (particle.jl:60-62: ρs0 / ρw0), and the
//     3D kernel writes mp.Δfs (utils_TS.jl:893-895): the fields meant are used;
//   * resetmpstatus_TS! evaluates the uGIMP basis on the first NIC of the
//     16 / 64 candidate nodes (utils_TS.jl:216-227, 266-283), leaving support
//     nodes out: the weights are the one-phase support-filtered stencil.
// Kept as written: grid.mi accumulates N·mw·n while the mixture's gravity uses
// the particle's mi = Ω((1-n)ρs + nρw); zero (not eps) guards the nodal
// inverses; the 3D G2P_TS! adds the solid strain increment to ϵijw.
//
// Same step structure as the one-phase MUSL kernels: particle masses ms = Ω·ρs
// and mw = Ω·ρw are invariant (Ω = JΩ0, ρ = ρ0/J) and kept per particle; the
// G2P pass carries DM1's position update and, fused, the next step's
// resetmpstatus_TS! + P2G_TS! at the new position.  Node records (FP32, 32 B):
//   acc  {ms, psx, psy, psz | fsx, fsy, fsz, mi}    gat  {vsT, 0 | vs -> Δus, 0}
//   accw {mw, pwx, pwy, pwz | fwx, fwy, fwz, 0}     gatw {vwT, 0 | vw -> Δuw, 0}
//   accd {fdx, fdy, fdz, 0}
#pragma once
#include "mpm_kernels.cuh"

namespace mpm {

// P2G_TS!, utils_TS.jl:295-393: solid mass (1-n)·ms, Σ N·mw·n, water mass,
// both momenta, the mixture force -Ω ∇N·(σ + σw I) + N·mi·G, the water force
// -Ω ∇N σw + N·mw·G (gravity on the last axis) and the drag N·(n mw G/k)(vw - vs).
template <int D, typename R>
__device__ __forceinline__ void p2g_scatter_ts(const GDev<R> &g, const AxisW<R> *w, R ms, R mw, R n, R vol,
                                               const R *vs, const R *vw, const R *s, R sw, R G, R kperm) {
    const MarkState mk = mark_begin<D, R>(g, w);
    const R one_n = R(1) - n;
    const R mi = one_n * ms + n * mw;   // Ω((1-n)ρs + nρw)
    const R tdg = (n * mw * G) / kperm;
    R ps[3], pw[3], dr[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        ps[d] = d < D ? ms * vs[d] * one_n : R(0);
        pw[d] = d < D ? mw * vw[d] * n : R(0);
        dr[d] = d < D ? tdg * (vw[d] - vs[d]) : R(0);
    }
    // rows of σ + σw I (Voigt xx yy zz xy yz zx; 2D xx yy zz xy)
    R sx[3], sy[3], sz[3];
    if (D == 2) {
        sx[0] = s[0] + sw; sx[1] = s[3]; sx[2] = R(0);
        sy[0] = s[3]; sy[1] = s[1] + sw; sy[2] = R(0);
        sz[0] = sz[1] = sz[2] = R(0);
    } else {
        sx[0] = s[0] + sw; sx[1] = s[3]; sx[2] = s[5];
        sy[0] = s[3]; sy[1] = s[1] + sw; sy[2] = s[4];
        sz[0] = s[5]; sz[1] = s[4]; sz[2] = s[2] + sw;
    }
    const int n0 = window_n0<D, R>(g, w);
    const int plane = g.nnx * g.nny;
    constexpr int NC = D == 3 ? 3 : 1;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        const R wz = D == 3 ? w[2].N[c] : R(1), gz = D == 3 ? w[2].dN[c] : R(0);
        if (wz == R(0)) continue;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const R wx = w[0].N[a], gx = w[0].dN[a];
            if (wx == R(0)) continue;
            const int col = n0 + a * g.nny + c * plane;
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                const R wy = w[1].N[b], gy = w[1].dN[b];
                if (wy == R(0)) continue;
                const R N = wx * wy * wz;
                const R dN[3] = {gx * wy * wz, wx * gy * wz, wx * wy * gz};
                R fs[3], fw[3];
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    fs[d] = R(0);
                    fw[d] = R(0);
                }
                fs[0] = -vol * (dN[0] * sx[0] + dN[1] * sx[1] + dN[2] * sx[2]);
                fs[1] = -vol * (dN[0] * sy[0] + dN[1] * sy[1] + dN[2] * sy[2]);
                if (D == 3) fs[2] = -vol * (dN[0] * sz[0] + dN[1] * sz[1] + dN[2] * sz[2]);
#pragma unroll
                for (int d = 0; d < D; ++d) fw[d] = -vol * (dN[d] * sw);
                fs[D - 1] += N * mi * G;
                fw[D - 1] += N * mw * G;
                const int q = col + b;
                red_add4(&g.acc[q].a, N * ms * one_n, N * ps[0], N * ps[1], N * ps[2]);
                red_add4(&g.acc[q].b, fs[0], fs[1], fs[2], N * mw * n);
                red_add4(&g.accw[q].a, N * mw, N * pw[0], N * pw[1], N * pw[2]);
                red_add4(&g.accw[q].b, fw[0], fw[1], fw[2], R(0));
                red_add4(&g.accd[q], N * dr[0], N * dr[1], N * dr[2], R(0));
            }
        }
    }
    mark_end<R>(g, mk);
}

template <int D, typename R>
__device__ __forceinline__ void load_vel(R *const *src, int64_t i, R *v) {
#pragma unroll
    for (int d = 0; d < 3; ++d) v[d] = d < D ? src[d][i] : R(0);
}

// Standalone two-phase P2G (first step after an upload).
template <int D, typename R>
__global__ void __launch_bounds__(256) k_p2g_ts(PDev<D, R> P, GDev<R> g, StepParams sp) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= sp.np) return;
    double x[3];
    load_x<D, R>(P, i, x);
    AxisW<R> w[3];
    if (!particle_weights<D, R>(x, g, w)) { atomicOr(g.err, ERR_OOG); return; }
    R vs[3], vw[3], s[6];
    load_vel<D, R>(P.v, i, vs);
    load_vel<D, R>(P.vw, i, vw);
#pragma unroll
    for (int k = 0; k < PDev<D, R>::NV; ++k) s[k] = P.sig[k][i];
    const Mat<R> &M = g.mat[P.mat[i]];
    p2g_scatter_ts<D, R>(g, w, P.m[i], P.mw[i], P.n[i], P.vol[i], vs, vw, s, P.sigw[i], (R)sp.G, M.kperm);
}

// solvegrid_TS!, utils_TS.jl:404-532.  Keeps the masses for DM3 and clears the
// momenta, forces, Σ N·mw·n and the drag.
template <int D, typename R>
__device__ __forceinline__ void solve_node_ts(const GDev<R> &g, const StepParams &sp, int i) {
    using T4 = typename Vec<R>::T4;
    const Node8<R> S = g.acc[i], W = g.accw[i];
    const T4 fd4 = g.accd[i];
    const R ms = S.a.x, mw = W.a.x, mi = S.b.w;
    const R msd = ms == R(0) ? R(0) : R(1) / ms, mwd = mw == R(0) ? R(0) : R(1) / mw;
    const R ps[3] = {S.a.y, S.a.z, S.a.w}, pw[3] = {W.a.y, W.a.z, W.a.w};
    const R fs[3] = {S.b.x, S.b.y, S.b.z}, fw[3] = {W.b.x, W.b.y, W.b.z}, fd[3] = {fd4.x, fd4.y, fd4.z};
    R vs[3] = {0, 0, 0}, vw[3] = {0, 0, 0}, vsT[3] = {0, 0, 0}, vwT[3] = {0, 0, 0};
    R qw = R(0), qs = R(0);
#pragma unroll
    for (int d = 0; d < D; ++d) {
        vs[d] = ps[d] * msd;
        vw[d] = pw[d] * mwd;
        qw += fw[d] * fw[d];
        qs += (fs[d] - fw[d]) * (fs[d] - fw[d]);
    }
    const R tw = -(R)sp.zeta_w * sqrt(qw), tsd = -(R)sp.zeta * sqrt(qs);
    const R dt = (R)sp.dt;
    const uint8_t bm = g.bcmask[i];
    R bv[3] = {0, 0, 0}, bw[3] = {0, 0, 0};
    if (g.bcval) { const T4 b = g.bcval[i]; bv[0] = b.x; bv[1] = b.y; bv[2] = b.z; }
    if (g.bcvalw) { const T4 b = g.bcvalw[i]; bw[0] = b.x; bw[1] = b.y; bw[2] = b.z; }
#pragma unroll
    for (int d = 0; d < D; ++d) {
        const R dw = tw * sgn(vw[d]), ds = tsd * sgn(vs[d]);
        const R aw = mwd * (fw[d] + dw + fd[d]);
        const R as = msd * (-mi * aw + fs[d] + dw + ds);
        vsT[d] = vs[d] + as * dt;
        vwT[d] = vw[d] + aw * dt;
        if (bm & (1 << d)) vsT[d] = bv[d];
        if (bm & (8 << d)) vwT[d] = bw[d];
    }
    Node8<R> o;
    o.a = mk4<R>(vsT[0], vsT[1], vsT[2], 0);
    o.b = mk4<R>(vs[0], vs[1], vs[2], 0);
    g.gat[i] = o;
    o.a = mk4<R>(vwT[0], vwT[1], vwT[2], 0);
    o.b = mk4<R>(vw[0], vw[1], vw[2], 0);
    g.gatw[i] = o;
    Node8<R> z;
    z.b = mk4<R>(0, 0, 0, 0);
    z.a = mk4<R>(ms, 0, 0, 0);
    g.acc[i] = z;
    z.a = mk4<R>(mw, 0, 0, 0);
    g.accw[i] = z;
    g.accd[i] = z.b;
}

template <int D, typename R>
__global__ void __launch_bounds__(128) k_solve_ts(GDev<R> g, StepParams sp) {
    const uint32_t nb = *g.bcount;
    for (uint32_t k = blockIdx.x; k < nb; k += gridDim.x) {
        const int i = block_node<D, R>(g, (int)g.blist[k], threadIdx.x);
        if (i >= 0) solve_node_ts<D, R>(g, sp, i);
    }
}

// doublemapping1_TS! (utils_TS.jl:543-648, velocities of both phases) fused
// with doublemapping2_TS! (utils_TS.jl:657-704, re-scatter of both momenta).
// The position update of DM1 is done by k_g2p_ts from the same ΣN·vsT.
// doublemapping1_TS! of one particle: gathers, both velocities (stored), both
// momenta for the re-scatter; w receives the particle's window.
template <int D, typename R>
__device__ __forceinline__ void dmap_ts_core(const PDev<D, R> &P, const GDev<R> &g, const StepParams &sp, int64_t i,
                                             AxisW<R> *w, R *ps, R *pw) {
    double x[3];
    load_x<D, R>(P, i, x);
    particle_weights<D, R>(x, g, w);   // out-of-grid particles get zero weights
    const int n0 = window_n0<D, R>(g, w);
    const int plane = g.nnx * g.nny;
    constexpr int NC = D == 3 ? 3 : 1;
    R s1[3] = {0, 0, 0}, s2[3] = {0, 0, 0}, w1[3] = {0, 0, 0}, w2[3] = {0, 0, 0};
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        const R wz = D == 3 ? w[2].N[c] : R(1);
        if (wz == R(0)) continue;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const R wxz = w[0].N[a] * wz;
            if (wxz == R(0)) continue;
            const int col = n0 + a * g.nny + c * plane;
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                const R wy = w[1].N[b];
                if (wy == R(0)) continue;
                const R N = wxz * wy;
                const Node8<R> S = g.gat[col + b], W = g.gatw[col + b];
                const R vT[3] = {S.a.x, S.a.y, S.a.z}, v0[3] = {S.b.x, S.b.y, S.b.z};
                const R wT[3] = {W.a.x, W.a.y, W.a.z}, w0[3] = {W.b.x, W.b.y, W.b.z};
#pragma unroll
                for (int d = 0; d < D; ++d) {
                    s1[d] += N * (vT[d] - v0[d]);
                    s2[d] += N * vT[d];
                    w1[d] += N * (wT[d] - w0[d]);
                    w2[d] += N * wT[d];
                }
            }
        }
    }
    const R FLIP = (R)sp.FLIP, PIC = (R)sp.PIC;
    const R n = P.n[i], ms = P.m[i], mw = P.mw[i];
    ps[0] = ps[1] = ps[2] = R(0);
    pw[0] = pw[1] = pw[2] = R(0);
#pragma unroll
    for (int d = 0; d < D; ++d) {
        const R vs = FLIP * (P.v[d][i] + s1[d]) + PIC * s2[d];
        const R vw = FLIP * (P.vw[d][i] + w1[d]) + PIC * w2[d];
        P.v[d][i] = vs;
        P.vw[d][i] = vw;
        ps[d] = ms * vs * (R(1) - n);
        pw[d] = mw * vw * n;
    }
}

// doublemapping1_TS! (utils_TS.jl:543-648, velocities of both phases) fused
// with doublemapping2_TS! (utils_TS.jl:657-704, re-scatter of both momenta).
// The position update of DM1 is done by k_g2p_ts from the same ΣN·vsT.
template <int D, typename R>
__global__ void __launch_bounds__(256) k_dmap_ts(PDev<D, R> P, GDev<R> g, StepParams sp) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= sp.np) return;
    AxisW<R> w[3];
    R ps[3], pw[3];
    dmap_ts_core<D, R>(P, g, sp, i, w, ps, pw);
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
            const int col = n0 + a * g.nny + c * plane;
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                const R wy = w[1].N[b];
                if (wy == R(0)) continue;
                const R N = wxz * wy;
                red_add4(&g.acc[col + b].a, R(0), N * ps[0], N * ps[1], N * ps[2]);
                red_add4(&g.accw[col + b].a, R(0), N * pw[0], N * pw[1], N * pw[2]);
            }
        }
    }
}

// The same pass (FP32) with the re-scatter of chained warp lanes merged (the
// momenta are lane constants, so only the weights are shuffled; see
// dm2_scatter_chain).
template <int D, typename R = float>
__global__ void __launch_bounds__(256, sizeof(R) == 8 ? MPM_CHAIN_MINB_F64 : MPM_TS_DMAP_CHAIN_MINB) k_dmap_ts_chain(PDev<D, R> P, GDev<R> g, StepParams sp) {
    // reverse block order, as k_dmap_chain: each pass starts on the particles
    // the previous pass touched last
    const int64_t i = (int64_t)(gridDim.x - 1 - blockIdx.x) * blockDim.x + threadIdx.x;
    const bool live = i < sp.np;
    AxisW<R> w[3];
    R ps[3] = {0, 0, 0}, pw[3] = {0, 0, 0};
    int n0 = 0, key = dead_key();
    if (live) {
        dmap_ts_core<D, R>(P, g, sp, i, w, ps, pw);
        n0 = key = window_n0<D, R>(g, w);
    } else {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            w[a].base = 0;
#pragma unroll
            for (int k = 0; k < 3; ++k) { w[a].N[k] = R(0.0); w[a].dN[k] = R(0.0); }
        }
    }
    const Chain ch = chain_of(key, g.nny);
    const unsigned F = 0xffffffffu;
    R s1[3], s2[3], q1[3], q2[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        s1[k] = __shfl_up_sync(F, ps[k], 1); s2[k] = __shfl_up_sync(F, ps[k], 2);
        q1[k] = __shfl_up_sync(F, pw[k], 1); q2[k] = __shfl_up_sync(F, pw[k], 2);
    }
    const int plane = g.nnx * g.nny;
    constexpr int NC = D == 3 ? 3 : 1;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        const R wz = D == 3 ? w[2].N[c] : R(1.0);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const R wxz = w[0].N[a] * wz;
            const R N0 = wxz * w[1].N[0], N1 = wxz * w[1].N[1], N2 = wxz * w[1].N[2];
            const R u1 = __shfl_up_sync(F, N1, 1), u2 = __shfl_up_sync(F, N2, 2), v2 = __shfl_up_sync(F, N2, 1);
            const R a1 = ch.c1 ? u1 : R(0.0), a2 = ch.c2 ? u2 : R(0.0), b2 = ch.c1 ? v2 : R(0.0);
            const int col = n0 + a * g.nny + c * plane;
            if (N0 + a1 + a2 != R(0.0)) {
                red_add4(&g.acc[col].a, R(0.0), N0 * ps[0] + a1 * s1[0] + a2 * s2[0], N0 * ps[1] + a1 * s1[1] + a2 * s2[1],
                         N0 * ps[2] + a1 * s1[2] + a2 * s2[2]);
                red_add4(&g.accw[col].a, R(0.0), N0 * pw[0] + a1 * q1[0] + a2 * q2[0],
                         N0 * pw[1] + a1 * q1[1] + a2 * q2[1], N0 * pw[2] + a1 * q1[2] + a2 * q2[2]);
            }
            if (ch.end) {
                if (N1 + b2 != R(0.0)) {
                    red_add4(&g.acc[col + 1].a, R(0.0), N1 * ps[0] + b2 * s1[0], N1 * ps[1] + b2 * s1[1],
                             N1 * ps[2] + b2 * s1[2]);
                    red_add4(&g.accw[col + 1].a, R(0.0), N1 * pw[0] + b2 * q1[0], N1 * pw[1] + b2 * q1[1],
                             N1 * pw[2] + b2 * q1[2]);
                }
                if (N2 != R(0.0)) {
                    red_add4(&g.acc[col + 2].a, R(0.0), N2 * ps[0], N2 * ps[1], N2 * ps[2]);
                    red_add4(&g.accw[col + 2].a, R(0.0), N2 * pw[0], N2 * pw[1], N2 * pw[2]);
                }
            }
        }
    }
}

// doublemapping3_TS!, utils_TS.jl:713-780: nodal velocities of both phases from
// the re-mapped momenta, BC, Δus = vs·ΔT, Δuw = vw·ΔT.  Clears the masses and
// momenta for the next P2G and the block flags.
template <int D, typename R>
__device__ __forceinline__ void dm3_node_ts(const GDev<R> &g, const StepParams &sp, int i) {
    using T4 = typename Vec<R>::T4;
    const T4 S = g.acc[i].a, W = g.accw[i].a;
    const R msd = S.x == R(0) ? R(0) : R(1) / S.x, mwd = W.x == R(0) ? R(0) : R(1) / W.x;
    const R ps[3] = {S.y, S.z, S.w}, pw[3] = {W.y, W.z, W.w};
    const uint8_t bm = g.bcmask[i];
    R bv[3] = {0, 0, 0}, bw[3] = {0, 0, 0};
    if (g.bcval) { const T4 b = g.bcval[i]; bv[0] = b.x; bv[1] = b.y; bv[2] = b.z; }
    if (g.bcvalw) { const T4 b = g.bcvalw[i]; bw[0] = b.x; bw[1] = b.y; bw[2] = b.z; }
    const R dt = (R)sp.dt;
    R us[3] = {0, 0, 0}, uw[3] = {0, 0, 0};
#pragma unroll
    for (int d = 0; d < D; ++d) {
        R vs = ps[d] * msd, vw = pw[d] * mwd;
        if (bm & (1 << d)) vs = bv[d];
        if (bm & (8 << d)) vw = bw[d];
        us[d] = vs * dt;
        uw[d] = vw * dt;
    }
    g.gat[i].b = mk4<R>(us[0], us[1], us[2], 0);
    g.gatw[i].b = mk4<R>(uw[0], uw[1], uw[2], 0);
    g.acc[i].a = mk4<R>(0, 0, 0, 0);
    g.accw[i].a = mk4<R>(0, 0, 0, 0);
}

template <int D, typename R>
__global__ void __launch_bounds__(128) k_dm3_ts(GDev<R> g, StepParams sp) {
    const uint32_t nb = *g.bcount;
    for (uint32_t k = blockIdx.x; k < nb; k += gridDim.x) {
        const int b = (int)g.blist[k];
        const int i = block_node<D, R>(g, b, threadIdx.x);
        if (i >= 0) dm3_node_ts<D, R>(g, sp, i);
        if (threadIdx.x == 0) g.bflag[b] = 0u;
    }
}

// G2P_TS! (utils_TS.jl:790-961): the solid part is G2P_OS!'s arithmetic
// (update_particle: position, strain, F, J, Ω, liE! + dpP!/mcP!), then the
// water strain, the pore pressure σw += Kw/n ((1-n) tr ΔFs + n tr ΔFw) and
// the porosity n = 1 - (1-n)/ΔJ with ΔJ = J Ω0 / Ω_old.  With FUSE the next
// step's P2G_TS! scatters the particle at its new position.
// G2P_TS! (utils_TS.jl:790-961) of one particle: the solid part is G2P_OS!'s
// arithmetic (update_particle: position, strain, F, J, Ω, liE! + dpP!/mcP!),
// then the water strain, the pore pressure σw += Kw/n ((1-n) tr ΔFs + n tr ΔFw)
// and the porosity n = 1 - (1-n)/ΔJ with ΔJ = J Ω0 / Ω_old.  Returns the new
// position x, stress s, volume vol, porosity nn and pore pressure sw_out.
template <int D, typename R, bool MC3>
__device__ __forceinline__ void g2p_ts_core(const PDev<D, R> &P, const GDev<R> &g, const StepParams &sp, int64_t i,
                                            double *x, AxisW<R> *w, R *s, R &vol, R &nn, R &sw_out, R &kperm,
                                            float *pre = nullptr) {
    load_x<D, R>(P, i, x);
    particle_weights<D, R>(x, g, w);
    const int n0 = window_n0<D, R>(g, w);
    const int plane = g.nnx * g.nny;
    constexpr int NC = D == 3 ? 3 : 1;
    // ΣΔu⊗∇N = Σ(Δu - Δu_c)⊗∇N (Σ∇N = 0): the window centre's increments are
    // subtracted so that FP32 sums of a near-translation do not cancel
    const int ncen = n0 + g.nny + 1 + (D == 3 ? plane : 0);
    const auto cs = g.gat[ncen].b, cw = g.gatw[ncen].b;
    R tT[3] = {0, 0, 0}, dF[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, dW[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        const R wz = D == 3 ? w[2].N[c] : R(1), gz = D == 3 ? w[2].dN[c] : R(0);
        if (wz == R(0)) continue;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const R wx = w[0].N[a], gx = w[0].dN[a];
            if (wx == R(0)) continue;
            const int col = n0 + a * g.nny + c * plane;
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                const R wy = w[1].N[b], gy = w[1].dN[b];
                if (wy == R(0)) continue;
                const R N = wx * wy * wz;
                const R dN[3] = {gx * wy * wz, wx * gy * wz, wx * wy * gz};
                const Node8<R> S = g.gat[col + b];
                const auto Wb = g.gatw[col + b].b;
                const R us[3] = {S.b.x - cs.x, S.b.y - cs.y, S.b.z - cs.z};
                const R uw[3] = {Wb.x - cw.x, Wb.y - cw.y, Wb.z - cw.z};
                tT[0] += N * S.a.x; tT[1] += N * S.a.y; tT[2] += N * S.a.z;
#pragma unroll
                for (int r = 0; r < D; ++r)
#pragma unroll
                    for (int q = 0; q < D; ++q) {
                        dF[r * D + q] += us[r] * dN[q];
                        dW[r * D + q] += uw[r] * dN[q];
                    }
            }
        }
    }
    const R vol_old = P.vol[i];
    double J = 1.0;
    if (pre) prefetch_wait();
    update_particle<D, R, MC3>(P, g, sp, i, x, tT, dF, s, vol, pre, &J);
    // water part of G2P_TS!
    const Mat<R> &M = g.mat[P.mat[i]];
    kperm = M.kperm;
    const R n = P.n[i];
    R trs, trw;
    if (D == 2) {
        P.epsw[0][i] += dW[0];
        P.epsw[1][i] += dW[3];
        P.epsw[3][i] += dW[1] + dW[2];
        trs = dF[0] + dF[3];
        trw = dW[0] + dW[3];
    } else {
        // the solid increments, as utils_TS.jl:929-934 writes them
        P.epsw[0][i] += dF[0];
        P.epsw[1][i] += dF[4];
        P.epsw[2][i] += dF[8];
        P.epsw[3][i] += dF[1] + dF[3];
        P.epsw[4][i] += dF[5] + dF[7];
        P.epsw[5][i] += dF[2] + dF[6];
        trs = dF[0] + dF[4] + dF[8];
        trw = dW[0] + dW[4] + dW[8];
    }
    const R dJ = (R)(J * (double)P.vol0[i] / (double)vol_old);
    const R sw = P.sigw[i] + (M.Kw / n) * ((R(1) - n) * trs + n * trw);
    nn = R(1) - (R(1) - n) / dJ;
    P.sigw[i] = sw_out = sw;
    P.n[i] = nn;
}

// G2P_TS! with, under FUSE, the next step's P2G_TS! at the particle's new position.
template <int D, typename R, bool FUSE, bool MC3 = false>
__global__ void __launch_bounds__(256) k_g2p_ts(PDev<D, R> P, GDev<R> g, StepParams sp) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= sp.np) return;
    double x[3];
    AxisW<R> w[3];
    R s[6], vol, nn, sw, kperm;
    g2p_ts_core<D, R, MC3>(P, g, sp, i, x, w, s, vol, nn, sw, kperm);
    if (FUSE) {
        if (!particle_weights<D, R>(x, g, w)) { atomicOr(g.err, ERR_OOG); return; }
        R vs[3], vw[3];
        load_vel<D, R>(P.v, i, vs);
        load_vel<D, R>(P.vw, i, vw);
        p2g_scatter_ts<D, R>(g, w, P.m[i], P.mw[i], nn, vol, vs, vw, s, sw, (R)sp.G, kperm);
    }
}

// P2G_TS! (FP32) with the records proportional to N -- solid mass and momentum,
// water mass and momentum, drag -- merged over chained warp lanes (their
// factors are lane constants, so the weights and those constants are
// shuffled; see dm2_scatter_chain); the force records, which depend on ∇N,
// are reduced per node as in p2g_scatter_ts.  The record groups are scattered
// in separate sweeps over the window, so only one group's factors are live at
// a time.  All lanes call it.
template <int D, typename R = float>
__device__ __forceinline__ void p2g_scatter_ts_chain(const GDev<R> &g, const AxisW<R> *w, int n0, int key,
                                                     R ms, R mw, R n, R vol, const R *vs,
                                                     const R *vw, const R *s, R sw, R G, R kperm) {
    const Chain ch = chain_of(key, g.nny);
    const R one_n = R(1.0) - n;
    const R mi = one_n * ms + n * mw;
    const R mwn = mw * n;
    // force records, per node: σ̃ = -Ω (σ + σw I) by rows, σ̃w = -Ω σw
    {
        const R swv = -vol * sw;
        R t[3][3];
        if (D == 2) {
            t[0][0] = -vol * s[0] + swv; t[0][1] = -vol * s[3]; t[0][2] = R(0.0);
            t[1][0] = -vol * s[3]; t[1][1] = -vol * s[1] + swv; t[1][2] = R(0.0);
            t[2][0] = t[2][1] = t[2][2] = R(0.0);
        } else {
            t[0][0] = -vol * s[0] + swv; t[0][1] = -vol * s[3]; t[0][2] = -vol * s[5];
            t[1][0] = -vol * s[3]; t[1][1] = -vol * s[1] + swv; t[1][2] = -vol * s[4];
            t[2][0] = -vol * s[5]; t[2][1] = -vol * s[4]; t[2][2] = -vol * s[2] + swv;
        }
        const int plane = g.nnx * g.nny;
        constexpr int NC = D == 3 ? 3 : 1;
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            const R wz = D == 3 ? w[2].N[c] : R(1.0), gz = D == 3 ? w[2].dN[c] : R(0.0);
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const R wx = w[0].N[a], gx = w[0].dN[a];
                const int col = n0 + a * g.nny + c * plane;
#pragma unroll
                for (int b = 0; b < 3; ++b) {
                    const R wy = w[1].N[b], gy = w[1].dN[b];
                    const R N = wx * wy * wz;
                    if (N == R(0.0)) continue;
                    const R dN[3] = {gx * wy * wz, wx * gy * wz, wx * wy * gz};
                    R fs[3], fw[3];
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        fs[k] = dN[0] * t[k][0] + dN[1] * t[k][1] + dN[2] * t[k][2];
                        fw[k] = k < D ? dN[k] * swv : R(0.0);
                    }
                    fs[D - 1] += N * mi * G;
                    fw[D - 1] += N * mw * G;
                    red_add4(&g.acc[col + b].b, fs[0], fs[1], fs[2], N * mwn);
                    red_add4(&g.accw[col + b].b, fw[0], fw[1], fw[2], R(0.0));
                }
            }
        }
    }
    // N-proportional records: acc.a = N·A, accw.a = N·B, accd = N·C
    {
        R A[4] = {ms * one_n, R(0.0), R(0.0), R(0.0)};
#pragma unroll
        for (int d = 0; d < D; ++d) A[1 + d] = ms * vs[d] * one_n;
        chain_nprop<D, 4>(g, w, n0, ch, A, [&](int i) { return &g.acc[i].a; });
    }
    {
        R B[4] = {mw, R(0.0), R(0.0), R(0.0)};
#pragma unroll
        for (int d = 0; d < D; ++d) B[1 + d] = mw * vw[d] * n;
        chain_nprop<D, 4>(g, w, n0, ch, B, [&](int i) { return &g.accw[i].a; });
    }
    {
        const R tdg = kperm != R(0.0) ? (n * mw * G) / kperm : R(0.0);
        R Cv[3] = {R(0.0), R(0.0), R(0.0)};
#pragma unroll
        for (int d = 0; d < D; ++d) Cv[d] = tdg * (vw[d] - vs[d]);
        chain_nprop<D, 3>(g, w, n0, ch, Cv, [&](int i) { return &g.accd[i]; });
    }
}

// The fused two-phase pass (FP32) with the lane-merged scatter.
template <int D, bool MC3 = false, typename R = float>
__global__ void __launch_bounds__(256, sizeof(R) == 8 ? MPM_TS_P_MINB_F64 : MPM_TS_P_MINB) k_g2p_ts_chain(PDev<D, R> P, GDev<R> g, StepParams sp) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    bool live = i < sp.np;
    double x[3];
    AxisW<R> w[3];
    R s[6] = {0, 0, 0, 0, 0, 0}, vol = 0, nn = 0, sw = 0, kperm = 0;
    R vs[3] = {0, 0, 0}, vw[3] = {0, 0, 0}, ms = 0, mw = 0;
    // FP32: the one-phase fields requested by cp.async before the gathers
    extern __shared__ float g2p_pre[];   // PF_N slots x 256 threads when sp.prefetch
    float *pre = nullptr;
    if (sizeof(R) == 4 && sp.prefetch && live) {
        pre = g2p_pre + threadIdx.x;
        prefetch_particle<D, R>(pre, P, i);
    }
    if (live) {
        g2p_ts_core<D, R, MC3>(P, g, sp, i, x, w, s, vol, nn, sw, kperm, pre);
        if (!particle_weights<D, R>(x, g, w)) {
            atomicOr(g.err, ERR_OOG);
            live = false;
        } else {
            load_vel<D, R>(P.v, i, vs);
            load_vel<D, R>(P.vw, i, vw);
            ms = P.m[i];
            mw = P.mw[i];
        }
    }
    int n0 = 0, key = dead_key();
    if (live) {
        n0 = key = window_n0<D, R>(g, w);
    } else {
        ms = mw = vol = R(0.0);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            w[a].base = 0;
#pragma unroll
            for (int k = 0; k < 3; ++k) { w[a].N[k] = R(0.0); w[a].dN[k] = R(0.0); }
        }
    }
    MarkState mk;
    if (live) mk = mark_begin<D, R>(g, w);
    p2g_scatter_ts_chain<D, R>(g, w, n0, key, ms, mw, nn, vol, vs, vw, s, sw, (R)sp.G, kperm);
    if (live) mark_end<R>(g, mk);
}

}  // namespace mpm
