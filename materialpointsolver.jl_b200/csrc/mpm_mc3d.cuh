// mpm_mc3d.cuh -- 3D Mohr-Coulomb stress return on the device (the "restated"
// mode of desc.mc3d).
//
// The reference's 3D mcP! body is commented out (src/materials/mohrcoulomb.jl:
// 152-455), so its literal 3D behaviour is the elastic predictor alone.  This
// file evaluates the algorithm that commented block describes: stress
// invariants (rho, theta, epsilon) of the trial stress, tension / shear
// classification with the apex criterion, flow direction from a hyperbolic
// (tension) or Menetrey-Willam (shear) potential, a first plastic corrector
// whose multiplier comes from the pre-increment stress when that stress sat on
// the surface (|f| < 0.1), else from the trial stress, then up to 100 further
// correctors until both yield functions are below 0.1.
//
// Always evaluated in FP64 whatever the precision of the rest of the step: the
// routine is branchy and transcendental-heavy but runs only on yielding
// particles, and FP64 keeps the acos / pow arguments well conditioned.
// __noinline__ keeps its registers out of the fused G2P kernel's budget.
#pragma once
#include <cuda_runtime.h>

namespace mpm {
namespace mc3d {

constexpr double PI = 3.141592653589793;
constexpr double EPS = 2.220446049250313e-16;   // machine epsilon of Float64
constexpr double TOL = 0.1;
constexpr int MAXIT = 100;
enum { ELASTIC = 0, TENSILE = 1, SHEAR = 2 };

struct Inv {
    double sm, j2, j3, rho, theta, epsilon;
    double dev[6];
};

__host__ __device__ __forceinline__ void invariants(const double *s, Inv &v) {
    const double sm = (s[0] + s[1] + s[2]) / 3.0;
    v.sm = sm;
    const double d0 = s[0] - sm, d1 = s[1] - sm, d2 = s[2] - sm;
    v.dev[0] = d0; v.dev[1] = d1; v.dev[2] = d2;
    v.dev[3] = s[3]; v.dev[4] = s[4]; v.dev[5] = s[5];
    const double j2 = ((s[0] - s[1]) * (s[0] - s[1]) + (s[1] - s[2]) * (s[1] - s[2]) +
                       (s[2] - s[0]) * (s[2] - s[0])) / 6.0 +
                      s[3] * s[3] + s[4] * s[4] + s[5] * s[5];
    const double j3 = d0 * d1 * d2 + 2.0 * s[3] * s[4] * s[5] - d0 * s[4] * s[4] - d1 * s[5] * s[5] -
                      d2 * s[3] * s[3];
    double lode = fabs(j2) > EPS ? (3.0 * sqrt(3.0) / 2.0) * (j3 / pow(j2, 1.5)) : 0.0;
    lode = fmin(1.0, fmax(-1.0, lode));
    v.j2 = j2;
    v.j3 = j3;
    v.theta = acos(lode) / 3.0;
    v.rho = sqrt(2.0 * j2);
    v.epsilon = sqrt(3.0) * sm;
}

struct Par {
    double K, G, c, phi, psi, st;
    double sphi, cphi, tphi, tpsi;
};

__host__ __device__ __forceinline__ int yield(const Inv &v, const Par &p, double &ft, double &fs) {
    const double r23 = sqrt(2.0 / 3.0), r15 = sqrt(1.5), r3 = sqrt(3.0);
    ft = r23 * cos(v.theta) * v.rho + v.epsilon / r3 - p.st;
    fs = r15 * v.rho * (sin(v.theta + PI / 3.0) / (r3 * p.cphi) + cos(v.theta + PI / 3.0) * p.tphi / 3.0) +
         (v.epsilon / r3) * p.tphi - p.c;
    if (ft > 0.0 && fs > 0.0) {
        // both violated: the apex criterion picks tension or shear
        const double nphi = (1.0 + p.sphi) / (1.0 - p.sphi);
        const double sp = p.st * nphi - 2.0 * p.c * sqrt(nphi);
        const double ap = sqrt(1.0 + nphi * nphi) + nphi;
        const double hh = ft + ap * (r23 * cos(v.theta - 4.0 * PI / 3.0) * v.rho + v.epsilon / r3 - sp);
        return hh > EPS ? TENSILE : SHEAR;
    }
    if (fs > 0.0) return SHEAR;
    if (ft > 0.0) return TENSILE;
    return ELASTIC;
}

// The two yield functions in FP32, for cheap acceptance tests of a stress
// that should lie on the surface (the surrogate's predictions): the same
// invariants and functions as invariants() and yield() above.
__device__ __forceinline__ void yield_f32(const float *s, const Par &p, float &ft, float &fs, float &sm_out) {
    const float sm = (s[0] + s[1] + s[2]) * (1.0f / 3.0f);
    const float d0 = s[0] - sm, d1 = s[1] - sm, d2 = s[2] - sm;
    const float j2 = (d0 * d0 + d1 * d1 + d2 * d2) * 0.5f + s[3] * s[3] + s[4] * s[4] + s[5] * s[5];
    const float j3 = d0 * d1 * d2 + 2.0f * s[3] * s[4] * s[5] - d0 * s[4] * s[4] - d1 * s[5] * s[5] -
                     d2 * s[3] * s[3];
    float lode = j2 > 1e-30f ? 2.598076211f * (j3 / (j2 * sqrtf(j2))) : 0.0f;
    lode = fminf(1.0f, fmaxf(-1.0f, lode));
    const float theta = acosf(lode) * (1.0f / 3.0f);
    const float rho = sqrtf(2.0f * j2), eps = 1.732050808f * sm;
    const float cphi = (float)p.cphi, tphi = (float)p.tphi;
    ft = 0.8164965809f * cosf(theta) * rho + eps * 0.5773502692f - (float)p.st;
    fs = 1.224744871f * rho *
             (sinf(theta + 1.047197551f) / (1.732050808f * cphi) + cosf(theta + 1.047197551f) * tphi * (1.0f / 3.0f)) +
         eps * 0.5773502692f * tphi - (float)p.c;
    sm_out = sm;
}

// FP32 screen of the classification, for skipping the FP64 invariants of
// clearly elastic stresses: true only when both yield functions, evaluated in
// FP32, lie below -0.02·(Σ|σ| + c + |σt|).  The FP32 evaluation errs by well
// under that: the invariants to a few ulp of the stress scale, and θ =
// acos(lode)/3 enters only through cos θ, sin(θ + π/3) and cos(θ + π/3), which
// are Hölder-1/2 in lode at lode = -1, so a lode error δ (≲ 1e-6·Σ|σ|/ρ) moves
// the ρ terms by ≲ ρ·sqrt(δ) ≤ 1.1e-3·Σ|σ|, times at most ~2.5 for the friction
// factors.  A screened stress is therefore ELASTIC in FP64 as well.  NaN or
// overflow fails the screen (the comparisons are false).
__device__ __forceinline__ bool surely_elastic(const double *s, const Par &p) {
    float sf[6], sa = 0.0f;
#pragma unroll
    for (int k = 0; k < 6; ++k) { sf[k] = (float)s[k]; sa += fabsf(sf[k]); }
    float ft, fs, sm;
    yield_f32(sf, p, ft, fs, sm);
    const float m = -0.02f * (sa + (float)p.c + fabsf((float)p.st));
    return ft < m && fs < m;
}

// df/dsigma, dg/dsigma (Voigt, engineering shear) and dg/dq for the given mode.
__host__ __device__ __forceinline__ void gradients(int type, const Inv &v, const Par &p, double *df, double *dg,
                                          double &dg_dq) {
    const double r23 = sqrt(2.0 / 3.0), r15 = sqrt(1.5), r3 = sqrt(3.0);
    const double th = v.theta, rho = v.rho;
    const double ct = cos(th), sn = sin(th);
    double df_de, df_dr, df_dt;
    if (type == TENSILE) {
        df_de = 1.0 / r3;
        df_dr = r23 * ct;
        df_dt = -r23 * rho * sn;
    } else {
        df_de = p.tphi / r3;
        df_dr = r15 * (sin(th + PI / 3.0) / (r3 * p.cphi) + cos(th + PI / 3.0) * p.tphi / 3.0);
        df_dt = r15 * rho * (cos(th + PI / 3.0) / (r3 * p.cphi) - sin(th + PI / 3.0) * p.tphi / 3.0);
    }
    // d(epsilon)/ds, d(rho)/ds, d(theta)/ds
    const double *d = v.dev;
    double dr_ds[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) dr_ds[k] = rho > EPS ? (k < 3 ? d[k] : 2.0 * d[k]) / rho : 0.0;
    double dj3[6];
    dj3[0] = d[0] * d[0] + d[3] * d[3] + d[5] * d[5] - 2.0 / 3.0 * v.j2;
    dj3[1] = d[3] * d[3] + d[1] * d[1] + d[4] * d[4] - 2.0 / 3.0 * v.j2;
    dj3[2] = d[5] * d[5] + d[4] * d[4] + d[2] * d[2] - 2.0 / 3.0 * v.j2;
    dj3[3] = 2.0 * (d[0] * d[3] + d[3] * d[1] + d[5] * d[4]);
    dj3[4] = 2.0 * (d[3] * d[5] + d[1] * d[4] + d[4] * d[2]);
    dj3[5] = 2.0 * (d[0] * d[5] + d[3] * d[4] + d[5] * d[2]);
    double dl_dj2 = -9.0 * sqrt(3.0) / 4.0 * v.j3, dl_dj3 = 3.0 * sqrt(3.0) / 2.0, dt_dl = -1.0 / 3.0;
    if (fabs(v.j2) > EPS) {
        const double r = v.j3 * 0.5 * pow(v.j2 / 3.0, -1.5);
        dl_dj2 *= pow(v.j2, -2.5);
        dl_dj3 *= pow(v.j2, -1.5);
        const double q = fabs(1.0 - r * r) < EPS ? EPS : fabs(1.0 - r * r);
        dt_dl = -1.0 / (3.0 * sqrt(q));
    }
    double dt_ds[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        const double dj2 = k < 3 ? d[k] : 2.0 * d[k];
        dt_ds[k] = dt_dl * (dl_dj2 * dj2 + dl_dj3 * dj3[k]);
    }
#pragma unroll
    for (int k = 0; k < 6; ++k) df[k] = (k < 3 ? df_de * (1.0 / r3) : 0.0) + df_dr * dr_ds[k] + df_dt * dt_ds[k];

    double dg_de, dg_dr, dg_dt;
    if (type == TENSILE) {
        // hyperbolic potential, eccentricity 0.6, apex distance 0.1 * sigma_t
        const double et = 0.6, xit = 0.1;
        double sq = 4.0 * (1.0 - et * et) * ct * ct + 5.0 * et * et - 4.0 * et;
        if (sq < EPS) sq = 0.00001;
        double den = 2.0 * (1.0 - et * et) * ct + (2.0 * et - 1.0) * sqrt(sq);
        const double num = 4.0 * (1.0 - et * et) * ct * ct + (2.0 * et - 1.0) * (2.0 * et - 1.0);
        if (den < EPS) den = 0.00001;
        const double rt = num / (3.0 * den);
        const double hyp = sqrt(xit * xit * p.st * p.st + 1.5 * rt * rt * rho * rho);
        const double dg_drt = 1.5 * rho * rho * rt / hyp;
        dg_dr = 1.5 * rho * rt * rt / hyp;
        dg_de = 1.0 / r3;
        const double dden_dt = -2.0 * (1.0 - et * et) * sn - (2.0 * et - 1.0) * 4.0 * (1.0 - et * et) * ct * sn / sqrt(sq);
        const double dnum_dt = -8.0 * (1.0 - et * et) * ct * sn;
        const double drt_dt = (dnum_dt * den - dden_dt * num) / (3.0 * den * den);
        dg_dt = dg_drt * drt_dt;
    } else {
        // Menetrey-Willam potential
        const double rmc = (3.0 - p.sphi) / (6.0 * p.cphi);
        double e = (3.0 - p.sphi) / (3.0 + p.sphi);
        if (e <= 0.5) e = 0.5000000001;
        else if (e > 1.0) e = 1.0;
        double sq = 4.0 * (1.0 - e * e) * ct * ct + 5.0 * e * e - 4.0 * e;
        if (sq < EPS) sq = 0.00001;
        double mm = 2.0 * (1.0 - e * e) * ct + (2.0 * e - 1.0) * sqrt(sq);
        if (mm < EPS) mm = 0.00001;
        const double l = 4.0 * (1.0 - e * e) * ct * ct + (2.0 * e - 1.0) * (2.0 * e - 1.0);
        const double rmw = (l / mm) * rmc;
        const double xi = 0.1;
        double om = (xi * p.c * p.tpsi) * (xi * p.c * p.tpsi) + (rmw * r15 * rho) * (rmw * r15 * rho);
        if (om < EPS) om = 0.00001;
        const double dl_dt = -8.0 * (1.0 - e * e) * ct * sn;
        const double dm_dt = -2.0 * (1.0 - e * e) * sn + 0.5 * (2.0 * e - 1.0) * dl_dt / sqrt(sq);
        const double drmw_dt = (mm * dl_dt - l * dm_dt) / (mm * mm);
        dg_de = p.tpsi / r3;
        dg_dr = 3.0 * rho * rmw * rmw / (2.0 * sqrt(om));
        dg_dt = 3.0 * rho * rho * rmw * rmc * drmw_dt / (2.0 * sqrt(om));
    }
#pragma unroll
    for (int k = 0; k < 6; ++k) dg[k] = (k < 3 ? dg_de * (1.0 / r3) : 0.0) + dg_dr * dr_ds[k] + dg_dt * dt_ds[k];
    dg_dq = dg_dr * r23;
}

// y = D_e x, isotropic elasticity with engineering shear
__host__ __device__ __forceinline__ void De_mul(const Par &p, const double *x, double *y) {
    const double Dt = p.K + 4.0 / 3.0 * p.G, Dd = p.K - 2.0 / 3.0 * p.G;
    y[0] = Dt * x[0] + Dd * x[1] + Dd * x[2];
    y[1] = Dd * x[0] + Dt * x[1] + Dd * x[2];
    y[2] = Dd * x[0] + Dd * x[1] + Dt * x[2];
    y[3] = p.G * x[3]; y[4] = p.G * x[4]; y[5] = p.G * x[5];
}

__host__ __device__ __forceinline__ double dot6(const double *a, const double *b) {
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2] + a[3] * b[3] + a[4] * b[4] + a[5] * b[5];
}

// s: trial stress (in/out); s0: rotated pre-increment stress; de: strain
// increment (engineering shear).  Returns whether the trial stress yielded
// (s changed) and the increment of the accumulated plastic shear strain epsq.
struct Ret {
    double dq;
    int yielded;
};
static __host__ __device__ __noinline__ Ret mohr_coulomb_3d(double *s, const double *s0, const double *de,
                                                            const Par p) {
    Inv v;
    double ft, fs;
    invariants(s, v);
    const int type_tr = yield(v, p, ft, fs);
    if (type_tr == ELASTIC) return Ret{0.0, 0};
    double df[6], dg[6], Ddf[6], Ddg[6], dq;
    gradients(type_tr, v, p, df, dg, dq);
    De_mul(p, df, Ddf);
    const double lam_tr = (type_tr == TENSILE ? ft : fs) / dot6(Ddf, dg);

    // the first corrector: multiplier from the pre-increment stress when it sat
    // on the surface, else from the trial stress
    Inv v0;
    double ft0, fs0;
    invariants(s0, v0);
    const int type0 = yield(v0, p, ft0, fs0);
    const double y0 = type0 == TENSILE ? ft0 : (type0 == SHEAR ? fs0 : 1.79769313486231570e308);
    double u[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) u[k] = s[k];
    double dpq;
    if (fabs(y0) < TOL) {
        double df0[6], dg0[6], dq0, Ddf0[6];
        gradients(type0, v0, p, df0, dg0, dq0);
        De_mul(p, df0, Ddf0);
        const double lam0 = dot6(Ddf0, de) / dot6(Ddf0, dg0);
        De_mul(p, dg0, Ddg);
#pragma unroll
        for (int k = 0; k < 6; ++k) u[k] -= lam0 * Ddg[k];
        dpq = lam0 * dq0;
    } else {
        De_mul(p, dg, Ddg);
#pragma unroll
        for (int k = 0; k < 6; ++k) u[k] -= lam_tr * Ddg[k];
        dpq = lam_tr * dq;
    }
    for (int it = 0; it < MAXIT; ++it) {
        invariants(u, v);
        const int t = yield(v, p, ft, fs);
        if (ft < TOL && fs < TOL) break;
        gradients(t, v, p, df, dg, dq);
        De_mul(p, df, Ddf);
        const double lam = (t == TENSILE ? ft : fs) / dot6(Ddf, dg);
        De_mul(p, dg, Ddg);
#pragma unroll
        for (int k = 0; k < 6; ++k) u[k] -= lam * Ddg[k];
        dpq += lam * dq;
    }
#pragma unroll
    for (int k = 0; k < 6; ++k) s[k] = u[k];
    return Ret{dpq, 1};
}

}  // namespace mc3d
}  // namespace mpm
