// mpm_device.cuh -- device-side building blocks of the uGIMP step:
// Julia-exact cell indexing, separable uGIMP weights, vector reductions and the
// per-particle constitutive update.  Citations are paths in the
// MaterialPointSolver.jl repository.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace mpm {

// sticky error bits (1 << -MPM_E_*)
constexpr int ERR_OOG = 1 << 3;   // stencil left the grid
constexpr int ERR_J = 1 << 4;     // det F <= 0
constexpr int ERR_NAN = 1 << 5;   // non-finite state
constexpr int ERR_OVF = 1 << 7;   // cell bucket too large for the sort

struct alignas(32) dvec4 { double x, y, z, w; };

template <typename R> struct Vec;
template <> struct Vec<float> { using T4 = float4; };
template <> struct Vec<double> { using T4 = dvec4; };

template <typename R> __device__ __forceinline__ typename Vec<R>::T4 mk4(R x, R y, R z, R w) {
    typename Vec<R>::T4 v; v.x = x; v.y = y; v.z = z; v.w = w; return v;
}

// ---------------------------------------------------------------------------
// reductions into global memory (relaxed, no return value)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void red_add4(float4 *a, float x, float y, float z, float w) {
    asm volatile("red.relaxed.gpu.global.add.v4.f32 [%0], {%1, %2, %3, %4};"
                 :: "l"(a), "f"(x), "f"(y), "f"(z), "f"(w) : "memory");
}
// The same reduction issued under a predicate instead of a branch: lanes whose
// contribution is zero (or that do not own the node) skip it without a
// divergent branch and its reconvergence point.  The address must be formed
// (it is not dereferenced when p is false).
__device__ __forceinline__ void red_add4_if(bool p, float4 *a, float x, float y, float z, float w) {
    asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %5, 0;\n\t"
                 "@q red.relaxed.gpu.global.add.v4.f32 [%0], {%1, %2, %3, %4};\n\t}"
                 :: "l"(a), "f"(x), "f"(y), "f"(z), "f"(w), "r"((unsigned)p) : "memory");
}
__device__ __forceinline__ void red_add4(dvec4 *a, double x, double y, double z, double w) {
    atomicAdd(&a->x, x); atomicAdd(&a->y, y); atomicAdd(&a->z, z);
    if (w != 0.0) atomicAdd(&a->w, w);
}
__device__ __forceinline__ void red_add4_if(bool p, dvec4 *a, double x, double y, double z, double w) {
    if (p) red_add4(a, x, y, z, w);
}

// ---------------------------------------------------------------------------
// Julia float fld / cld (div with RoundDown / RoundUp): round((a - mod(a, ±b)) / b),
// with Julia's float mod (rem = fmod, then shifted to the divisor's sign).
// Used by p2c, src/solvers/utils_OS.jl:203-205, 325-328.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double jl_mod(double x, double y) {
    double r = fmod(x, y);
    if (r == 0.0) return copysign(r, y);
    if ((r > 0.0) != (y > 0.0)) return __dadd_rn(r, y);
    return r;
}
__device__ __forceinline__ double jl_fld(double a, double b) {
    return rint(__ddiv_rn(__dsub_rn(a, jl_mod(a, b)), b));
}
__device__ __forceinline__ double jl_cld(double a, double b) {
    return rint(__ddiv_rn(__dsub_rn(a, jl_mod(a, -b)), b));
}
// clamp a float cell quotient into int range (NaN -> huge negative)
__device__ __forceinline__ int q2i(double q) {
    if (!(q >= -1.0e9)) return -1000000000;
    if (q > 1.0e9) return 1000000000;
    return (int)q;
}

template <typename R> __device__ __forceinline__ R sgn(R x) { return (R)((x > R(0)) - (x < R(0))); }

// ---------------------------------------------------------------------------
// Per-axis constants of the uGIMP basis (mpbasisfunc.jl:40-120).
// ---------------------------------------------------------------------------
template <typename R> struct AxisC {
    double x1, h;       // grid origin / spacing (FP64, for distances)
    double inv_h;       // 1/h (FP64) for the fast cell index
    double supp;        // h + lp/2: candidate test |Δ| < supp (utils_OS.jl:220-221)
    R hr, lp, half_lp, h_m_hl, h_p_hl;   // h, lp, lp/2, h - lp/2, h + lp/2
    R invhl, invh;                       // 1/(h lp), 1/h
    int nn, nc;         // nodes / cells on this axis
};

// 1-D uGIMP weight and derivative.  FP64 mode evaluates the CPU (division)
// form of uGIMPbasis piece by piece; FP32 mode the same function (the
// reciprocal form of uGIMPbasisx/y/z, |Δ|/h taken as |Δ|·(1/h)) written
// without branches, so the lanes of a warp whose particles fall in different
// pieces do not diverge (9 evaluations per window, two windows per particle in
// the fused pass).
template <typename R> __device__ __forceinline__ void ugimp1(R d, const AxisC<R> &c, R &N, R &dN) {
    R a = fabs(d);
    N = R(0); dN = R(0);
    if (sizeof(R) == 8) {
        R h = c.hr, lp = c.lp;
        if (a < R(0.5) * lp) {
            N = R(1) - ((R(4) * d * d + lp * lp) / (R(4) * h * lp));
            dN = -((R(8) * d) / (R(4) * h * lp));
        } else if (a < (h - R(0.5) * lp)) {
            N = R(1) - (a / h);
            dN = sgn(d) * (R(-1) / h);
        } else if (a < (h + R(0.5) * lp)) {
            R t = h + R(0.5) * lp - a;
            N = (t * t) / (R(2) * h * lp);
            dN = -sgn(d) * (t / (h * lp));
        }
    } else {
        // branch-free: the hat 1 - a/h with its kinks at 0 and at h smoothed over
        // the particle length lp (the three pieces of uGIMPbasisx/y/z in one
        // expression: -u0²/(h·lp) for a < lp/2, +u1²/(2h·lp) for a > h - lp/2)
        const R u0 = fmax(c.half_lp - a, R(0)), u1 = fmax(a - c.h_m_hl, R(0));
        const R in = a < c.h_p_hl ? R(1) : R(0);
        N = in * (R(1) - a * c.invh - u0 * u0 * c.invhl + R(0.5) * u1 * u1 * c.invhl);
        const R da = -c.invh + (R(2) * u0 + u1) * c.invhl;   // dN/d|Δ|
        dN = in * (d < R(0) ? -da : da);
    }
}

// The three window nodes of one axis.  With lp <= h at most three nodes lie in
// the support |Δ| < h + lp/2 and they are consecutive: node ci - 1 can only be
// in it when the particle sits in the lower half of its cell (offset below
// h/2, as lp/2 <= h/2), node ci + 2 only in the upper half.  The window is
// ci - 1 .. ci + 1 for the lower half and ci .. ci + 2 for the upper one; the
// node it adds beyond the support carries weight 0.  Splitting at the cell
// centre (rather than at the support edge h - lp/2 from the node) keeps the
// window of a particle on the regular lattice positions (h/4, 3h/4 for two per
// cell) fixed under small motions, so particles of one sub-cell octant share
// a window shape.  Nodes outside the grid get weight 0 and raise the
// out-of-grid flag when they would have carried weight.
// offset of a particle from node ci of its cell, in FP64 without contraction
// (the cell sort classifies sub-cell octants with the same expression)
template <typename R> __device__ __forceinline__ double cell_offset(double xp, int ci, const AxisC<R> &c) {
    return __dsub_rn(xp, __dadd_rn(c.x1, __dmul_rn((double)ci, c.h)));
}

template <typename R> struct AxisW {
    int base;
    R N[3], dN[3];
};

template <typename R>
__device__ __forceinline__ bool axis_weights(double xp, int ci, const AxisC<R> &c, AxisW<R> &w) {
    // distances to nodes ci-1 .. ci+1 (or ci .. ci+2) from the offset to node ci
    const double s = cell_offset(xp, ci, c);
    const int lo = s < 0.5 * c.h ? 1 : 0;
    const int base = ci - lo;
    bool oob = false;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double d = s + (double)(lo - k) * c.h;
        R n, dn;
        ugimp1<R>((R)d, c, n, dn);
        w.N[k] = n; w.dN[k] = dn;
    }
    w.base = base;
    if (base < 0 || base + 2 >= c.nn) {
        // Window reaches past the grid (rare).  A node outside the grid with
        // weight is an error.  A weightless one past the far end is traded for
        // the weightless node ci - 1, so that every valid window lies inside
        // the grid and its nodes can be read without guards.
        bool heavy = false;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            int j = base + k;
            if ((j < 0 || j >= c.nn) && w.N[k] != R(0)) heavy = true;
        }
        if (heavy || base < 0) {
            oob = true;
        } else {   // lo == 0: node ci - 1 = base - 1 is outside the support
            w.base = base - 1;
            w.N[2] = w.N[1]; w.dN[2] = w.dN[1];
            w.N[1] = w.N[0]; w.dN[1] = w.dN[0];
            w.N[0] = R(0); w.dN[0] = R(0);
            if (w.base < 0) oob = true;
        }
    }
    return oob;
}

// Cell index with Julia's fld (x, z) / cld - 1 (y) semantics.  Away from an
// integer quotient, floor((x - x1) * (1/h)) is the exact answer (the FP64
// quotient is within 1e-9 cell of the exact one for grids below ~1e6 cells per
// axis); within 1e-9 of an integer the exact-remainder rule decides.
template <typename R> __device__ __forceinline__ int cell_fld(double x, const AxisC<R> &c) {
    const double a = x - c.x1;
    const double t = a * c.inv_h;
    const double q = floor(t);
    const double fr = t - q;
    if (fr > 1e-9 && fr < 1.0 - 1e-9 && fabs(q) < 1.0e9) return (int)q;
    return q2i(jl_fld(a, c.h));
}
template <typename R> __device__ __forceinline__ int cell_cld_m1(double x, const AxisC<R> &c) {
    const double a = x - c.x1;
    const double t = a * c.inv_h;
    const double q = floor(t);
    const double fr = t - q;
    if (fr > 1e-9 && fr < 1.0 - 1e-9 && fabs(q) < 1.0e9) return (int)q;   // ceil(t) - 1
    return q2i(jl_cld(a, c.h)) - 1;
}

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// ---------------------------------------------------------------------------
// Material constants, precomputed on the host from Property (property.jl:31-53).
// ---------------------------------------------------------------------------
template <typename R> struct Mat {
    R K, G, Dt, Dd;                 // Dt = K + 1.333333 G, Dd = K - 0.666667 G (linearelastic.jl:48-49)
    R c, phi, psi, sigt, Hp, cr;
    R kphi, qphi, qpsi, st, ab, tb, dq;   // Drucker-Prager (druckerprager.jl:39-44, 59)
    R sphi, cphi, tphi, spsi, tpsi;       // Mohr-Coulomb
    R kc;                                 // kphi per unit cohesion
    R Kw, kperm;                          // two-phase: water bulk modulus, permeability k
    R pad[3];
};

// liE!, src/materials/linearelastic.jl:22-69 (2D) / :78-140 (3D).  s: Voigt
// stress (in/out), dF: incremental deformation gradient (row-major), de: strain
// increment (engineering shear).  s_rot receives the rotated pre-increment stress.
template <int D, typename R>
__device__ __forceinline__ void lin_elastic(R *s, const R *dF, const R *de, const Mat<R> &M, R *s_rot) {
    if (D == 2) {
        R w = R(0.5) * (dF[1] - dF[2]);
        R s1 = s[0], s2 = s[1], s4 = s[3];
        s[0] += w * s4 * R(2);
        s[1] += -w * s4 * R(2);
        s[3] += w * (s2 - s1);
    } else {
        R wxy = R(0.5) * (dF[3] - dF[1]);
        R wyz = R(0.5) * (dF[7] - dF[5]);
        R wxz = R(0.5) * (dF[6] - dF[2]);
        R s1 = s[0], s2 = s[1], s3 = s[2], s4 = s[3], s5 = s[4], s6 = s[5];
        s[0] += R(2) * (s4 * wxy + s6 * wxz);
        s[1] += -R(2) * (s4 * wxy - s5 * wyz);
        s[2] += -R(2) * (s6 * wxz + s5 * wyz);
        s[3] += wxy * (s2 - s1) + wxz * s5 + wyz * s6;
        s[4] += wyz * (s3 - s2) - wxz * s4 - wxy * s6;
        s[5] += wxz * (s3 - s1) + wxy * s5 - wyz * s4;
    }
    constexpr int NV = D == 2 ? 4 : 6;
#pragma unroll
    for (int k = 0; k < NV; ++k) s_rot[k] = s[k];
    s[0] += M.Dt * de[0] + M.Dd * de[1] + M.Dd * de[2];
    s[1] += M.Dd * de[0] + M.Dt * de[1] + M.Dd * de[2];
    s[2] += M.Dd * de[0] + M.Dd * de[1] + M.Dt * de[2];
    s[3] += M.G * de[3];
    if (D == 3) { s[4] += M.G * de[4]; s[5] += M.G * de[5]; }
}

// dpP!, src/materials/druckerprager.jl:22-80 (2D) / :89-155 (3D); sm, sij are
// the mean / deviatoric stress of the elastic predictor (liE! epilogue).
template <int D, typename R>
__device__ __forceinline__ void drucker_prager(R *s, R &epsq, R &epsk, const Mat<R> &M) {
    constexpr int NV = D == 2 ? 4 : 6;
    R sm = (s[0] + s[1] + s[2]) * R(0.333333);
    R sij[NV];
    sij[0] = s[0] - sm; sij[1] = s[1] - sm; sij[2] = s[2] - sm;
#pragma unroll
    for (int k = 3; k < NV; ++k) sij[k] = s[k];
    R tt = R(0.5) * (sij[0] * sij[0] + sij[1] * sij[1] + sij[2] * sij[2]) + sij[3] * sij[3];
    if (D == 3) tt += sij[4] * sij[4] + sij[5] * sij[5];
    R tau = sqrt(tt);
    R fs = tau + M.qphi * sm - M.kphi;
    R ft = sm - M.st;
    R BF = (tau - M.tb) - (M.ab * (sm - M.st));
    if (((sm < M.st) && (fs > R(0))) || ((sm >= M.st) && (BF > R(0)))) {
        R dl = fs / (M.G + M.K * M.qphi * M.qpsi);
        R t1 = sm - M.K * M.qpsi * dl;
        R t2 = (M.kphi - M.qphi * t1) / tau;
        s[0] = sij[0] * t2 + t1;
        s[1] = sij[1] * t2 + t1;
        s[2] = sij[2] * t2 + t1;
#pragma unroll
        for (int k = 3; k < NV; ++k) s[k] = sij[k] * t2;
        epsq += dl * M.dq;
        epsk += dl * M.qpsi;
    }
    if ((sm >= M.st) && (BF <= R(0))) {
        R dl = ft / M.K;
        s[0] = sij[0] + M.st;
        s[1] = sij[1] + M.st;
        s[2] = sij[2] + M.st;
        epsq += dl * R(0.333333) * R(1.414214);
        epsk += dl;
    }
}

// mcP! 2D, src/materials/mohrcoulomb.jl:22-86 (in-plane Mohr-Coulomb).
template <typename R>
__device__ __forceinline__ void mohr_coulomb_2d(R *s, R &epsq, R &epsk, const Mat<R> &M) {
    R c = fmax(M.c + M.Hp * epsq, M.cr);
    R ds = s[0] - s[1];
    R tau = sqrt(R(0.25) * ds * ds + s[3] * s[3]);
    R sig = R(0.5) * (s[0] + s[1]);
    R f = tau + sig * M.sphi - c * M.cphi;
    R sn1 = s[0], sn2 = s[1], sn3 = s[2], sn4 = s[3];
    R dsigB = c / M.tphi;
    if ((sig <= dsigB) && (f > R(0))) {
        R beta = fabs(c * M.cphi - sig * M.sphi) / tau;
        R dsigA = R(0.5) * beta * ds;
        sn1 = sig + dsigA;
        sn2 = sig - dsigA;
        sn4 = beta * s[3];
    }
    if ((sig > dsigB) && (f > R(0))) { sn1 = dsigB; sn2 = dsigB; sn4 = R(0); }
    R d1 = sn1 - s[0], d2 = sn2 - s[1], d3 = sn3 - s[2], d4 = sn4 - s[3];
    s[0] = sn1; s[1] = sn2; s[2] = sn3; s[3] = sn4;
    R base = R(1) / ((M.Dd - M.Dt) * (R(2) * M.Dd + M.Dt));
    R exx = -(M.Dd * d1 + M.Dt * d1 - M.Dd * d2 - M.Dd * d3) * base;
    R eyy = -(-M.Dd * d1 + M.Dd * d2 + M.Dt * d2 - M.Dd * d3) * base;
    R ezz = -(-M.Dd * d1 - M.Dd * d2 + M.Dd * d3 + M.Dt * d3) * base;
    R exy = d4 / M.G;
    epsk = exx + eyy + ezz;
    epsq += sqrt(R(0.666667) * (exx * exx + eyy * eyy + ezz * ezz + exy * exy * R(2)));
}

}  // namespace mpm
