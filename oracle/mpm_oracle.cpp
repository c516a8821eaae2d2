// mpm_oracle.cpp -- FP64 CPU restatement of MaterialPointSolver.jl v0.3.0's
// one-phase explicit uGIMP step (OS / MUSL, va = :a and :v).
//
// TEST INFRASTRUCTURE ONLY.  tests/, bench.py's cpu_baseline / reference arm and
// __graft_entry__.smoke() use it as the checker.  The product (libmpm_b200.so)
// never links or calls it.
//
// Parity status: UNPINNED by the reference (Julia is not installed here and the
// reference's tests pin no numbers).  Cross-checked by hand-derived known-answer
// tests and an independent pure-Python transliteration (tests/oracle_py.py).
//
// Every function follows the reference CPU path line by line, keeping its
// decimal constants (0.333333, 1.333333, 0.666667, 1.732051, ...), its candidate
// stencil order and its summation order (sequential mode, nthreads <= 1).
// File:line citations are relative to the MaterialPointSolver.jl repository.
#include "mpm_oracle.h"
#include <cmath>
#include <vector>
#include <cstring>
#include <cfloat>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

inline double sgn(double x) { return (x > 0.0) - (x < 0.0); }   // Julia sign()

// eps(T2) of the solves' massless-node cutoff (utils_OS.jl:515, 555, 975), T2
// the reference's float type
inline double mass_eps(const orc_model *m) { return m->f32 ? (double)FLT_EPSILON : DBL_EPSILON; }

// Julia `mod(x, y)` for floats (base/float.jl): r = rem(x,y); fix sign to y's.
inline double jl_mod(double x, double y) {
    double r = std::fmod(x, y);
    if (r == 0.0) return std::copysign(r, y);
    if ((r > 0.0) != (y > 0.0)) return r + y;
    return r;
}

// Integer ceil division for positive integers (Julia cld on Int).
inline int64_t icld(int64_t a, int64_t b) {
    int64_t q = a / b;
    if ((a % b != 0) && ((a > 0) == (b > 0))) q += 1;
    return q;
}

// 2D uGIMP candidate stencil grid.p2nD for NIC = 9 (src/types/grid.jl:132-137):
// rows {a, b} with a in {-nny, 0, nny, 2nny} (column shift) and b in {2,1,0,-1}.
void p2nD_2d(int64_t nny, int64_t tab[16][2]) {
    const int64_t a[4] = {-nny, 0, nny, 2 * nny};
    const int64_t b[4] = {2, 1, 0, -1};
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) { tab[i * 4 + j][0] = a[i]; tab[i * 4 + j][1] = b[j]; }
}

// 3D uGIMP candidate stencil grid.p2nD for NIC = 27 (src/types/grid.jl:289-301),
// 64 rows of (layer shift, column shift, row shift, extra row shift).  The
// order is the reference's; it fixes which candidate lands in which slot.
const int64_t P2ND_3D[64][4] = {
    {-1,-1,-1,0},{-1,0,-1,0},{0,0,-1,0},{0,-1,-1,0},{0,-2,-1,0},{-1,-2,-1,0},
    {-2,-2,-1,0},{-2,-1,-1,0},{-2,0,-1,0},{-2,1,-1,0},{-1,1,-1,0},{0,1,-1,0},
    {1,1,-1,0},{1,0,-1,0},{1,-1,-1,0},{1,-2,-1,0},{-1,-1,-1,1},{-1,0,-1,1},
    {0,0,-1,1},{0,-1,-1,1},{0,-2,-1,1},{-1,-2,-1,1},{-2,-2,-1,1},{-2,-1,-1,1},
    {-2,0,-1,1},{-2,1,-1,1},{-1,1,-1,1},{0,1,-1,1},{1,1,-1,1},{1,0,-1,1},
    {1,-1,-1,1},{1,-2,-1,1},{-1,-1,0,1},{-1,0,0,1},{0,0,0,1},{0,-1,0,1},
    {0,-2,0,1},{-1,-2,0,1},{-2,-2,0,1},{-2,-1,0,1},{-2,0,0,1},{-2,1,0,1},
    {-1,1,0,1},{0,1,0,1},{1,1,0,1},{1,0,0,1},{1,-1,0,1},{1,-2,0,1},
    {-1,-1,0,2},{-1,0,0,2},{0,0,0,2},{0,-1,0,2},{0,-2,0,2},{-1,-2,0,2},
    {-2,-2,0,2},{-2,-1,0,2},{-2,0,0,2},{-2,1,0,2},{-1,1,0,2},{0,1,0,2},
    {1,1,0,2},{1,0,0,2},{1,-1,0,2},{1,-2,0,2}};

// getP2N_uGIMP 2D, src/toolkits/p2nindex.jl:130-140 (1-based node id)
inline int64_t getP2N_2d(const orc_model *m, int64_t p2c, const int64_t tab[16][2], int iy) {
    int64_t col = icld(p2c, m->ncy);
    int64_t row = p2c - (col - 1) * m->ncy;
    int64_t ltn = col * m->nny - row;
    return ltn + tab[iy][0] + tab[iy][1];
}

// getP2N_uGIMP 3D, src/toolkits/p2nindex.jl:243-255 (1-based node id)
inline int64_t getP2N_3d(const orc_model *m, int64_t p2c, int iy) {
    int64_t layer = icld(p2c, m->ncx * m->ncy);
    int64_t l_idx = icld(p2c - (layer - 1) * m->ncx * m->ncy, m->ncy);
    int64_t l_idy = (p2c - (layer - 1) * m->ncx * m->ncy) - (l_idx - 1) * m->ncy;
    const int64_t *t = P2ND_3D[iy];
    return (layer + t[0]) * m->nnx * m->nny + (l_idx + t[1]) * m->nny + (l_idy + t[2]) + t[3];
}

inline int nv_of(int dim) { return dim == 2 ? 4 : 6; }

inline bool par(const orc_model *m) { return m->nthreads > 1; }

inline void atomic_add(double *a, double v, bool atomic) {
    if (atomic) {
#pragma omp atomic
        *a += v;
    } else {
        *a += v;
    }
}

}  // namespace

extern "C" {

// Julia `fld(a, b) = div(a, b, RoundDown) = round((a - mod(a, b)) / b)`:
// the exact-remainder rule, which differs from floor(a/b) when a/b rounds
// across an integer.
double orc_fld(double a, double b) { return std::nearbyint((a - jl_mod(a, b)) / b); }
// Julia `cld(a, b) = div(a, b, RoundUp) = round((a - mod(a, -b)) / b)`.
double orc_cld(double a, double b) { return std::nearbyint((a - jl_mod(a, -b)) / b); }

// uGIMPbasis, src/toolkits/mpbasisfunc.jl:40-53 (the CPU form with divisions).
void orc_ugimp(double d, double h, double lp, double *Np, double *dNp) {
    double Ni = 0.0, dN = 0.0, a = std::fabs(d);
    if (a < 0.5 * lp) {
        Ni = 1.0 - ((4.0 * d * d + lp * lp) / (4.0 * h * lp));
        dN = -((8.0 * d) / (4.0 * h * lp));
    } else if ((0.5 * lp) <= a && a < (h - 0.5 * lp)) {
        Ni = 1.0 - (a / h);
        dN = sgn(d) * (-1.0 / h);
    } else if ((h - 0.5 * lp) <= a && a < (h + 0.5 * lp)) {
        Ni = ((h + 0.5 * lp - a) * (h + 0.5 * lp - a)) / (2.0 * h * lp);
        dN = -sgn(d) * ((h + 0.5 * lp - a) / (h * lp));
    }
    *Np = Ni;
    *dNp = dN;
}

// p2c, utils_OS.jl:247-249 (2D) and :380-383 (3D); unsafe_trunc of a float sum.
void orc_p2c(const orc_model *m, const double *xi, int64_t np, int64_t *out) {
    for (int64_t i = 0; i < np; ++i) {
        double x = xi[i], y = xi[i + np];
        double v;
        if (m->dim == 2) {
            v = orc_cld(y - m->y1, m->dy) + orc_fld(x - m->x1, m->dx) * (double)m->ncy;
        } else {
            double z = xi[i + 2 * np];
            v = orc_cld(y - m->y1, m->dy) +
                orc_fld(z - m->z1, m->dz) * (double)m->ncy * (double)m->ncx +
                orc_fld(x - m->x1, m->dx) * (double)m->ncy;
        }
        out[i] = (int64_t)std::trunc(v);
    }
}

// resetgridstatus_OS!, utils_OS.jl:58-99
void orc_resetgrid(orc_model *m) {
    const int64_t ni = m->ni, D = m->dim;
    for (int64_t i = 0; i < ni; ++i) {
        if (i < m->nc) { m->g_sigm[i] = 0.0; m->g_omega[i] = 0.0; }
        m->g_ms[i] = 0.0;
        for (int d = 0; d < D; ++d) { m->g_ps[i + ni * d] = 0.0; m->g_fs[i + ni * d] = 0.0; }
        if (m->coupling == 1) {   // resetgridstatus_TS!, utils_TS.jl:44-106
            m->g_mi[i] = 0.0;
            m->g_mw[i] = 0.0;
            for (int d = 0; d < D; ++d) {
                m->g_pw[i + ni * d] = 0.0;
                m->g_fw[i + ni * d] = 0.0;
                m->g_fd[i + ni * d] = 0.0;
            }
        }
    }
}

// resetmpstatus_OS_CPU!, utils_OS.jl:235-277 (2D) and :363-415 (3D)
void orc_resetmp(orc_model *m) {
    const int64_t np = m->np, NIC = m->nic;
    const int D = m->dim;
    int64_t tab2[16][2];
    if (D == 2) p2nD_2d(m->nny, tab2);
    const int64_t ni = m->ni;
#pragma omp parallel for if (par(m)) schedule(static)
    for (int64_t ix = 0; ix < np; ++ix) {
        double mpms = m->Omega[ix] * m->rho[ix];
        m->ms[ix] = mpms;
        for (int d = 0; d < D; ++d) m->ps[ix + np * d] = mpms * m->vs[ix + np * d];
        double x = m->xi[ix], y = m->xi[ix + np];
        double v;
        if (D == 2) {
            v = orc_cld(y - m->y1, m->dy) + orc_fld(x - m->x1, m->dx) * (double)m->ncy;
        } else {
            double z = m->xi[ix + 2 * np];
            v = orc_cld(y - m->y1, m->dy) +
                orc_fld(z - m->z1, m->dz) * (double)m->ncy * (double)m->ncx +
                orc_fld(x - m->x1, m->dx) * (double)m->ncy;
        }
        int64_t p2c = (int64_t)std::trunc(v);
        m->p2c[ix] = p2c;
        for (int64_t s = 0; s < NIC; ++s) {
            m->Nij[ix + np * s] = 0.0;
            m->dNx[ix + np * s] = 0.0;
            m->dNy[ix + np * s] = 0.0;
            if (D == 3) m->dNz[ix + np * s] = 0.0;
        }
        int64_t viy = 1;
        const int ncand = D == 2 ? 16 : 64;
        for (int iy = 0; iy < ncand; ++iy) {
            int64_t p2n = D == 2 ? getP2N_2d(m, p2c, tab2, iy) : getP2N_3d(m, p2c, iy);
            int64_t n0 = p2n - 1;
            double ddx = x - m->g_xi[n0];
            double ddy = y - m->g_xi[n0 + ni];
            if (D == 2) {
                if (std::fabs(ddx) < (m->dx + 0.5 * m->lpx) &&
                    std::fabs(ddy) < (m->dy + 0.5 * m->lpy)) {
                    double Nx, dNx, Ny, dNy;
                    orc_ugimp(ddx, m->dx, m->lpx, &Nx, &dNx);
                    orc_ugimp(ddy, m->dy, m->lpy, &Ny, &dNy);
                    int64_t s = viy - 1;
                    m->Nij[ix + np * s] = Nx * Ny;
                    m->dNx[ix + np * s] = dNx * Ny;
                    m->dNy[ix + np * s] = dNy * Nx;
                    m->p2n[ix + np * s] = p2n;
                    viy += 1;
                }
            } else {
                double z = m->xi[ix + 2 * np];
                double ddz = z - m->g_xi[n0 + 2 * ni];
                if (std::fabs(ddx) < (m->dx + 0.5 * m->lpx) &&
                    std::fabs(ddy) < (m->dy + 0.5 * m->lpy) &&
                    std::fabs(ddz) < (m->dz + 0.5 * m->lpz)) {
                    double Nx, dNx, Ny, dNy, Nz, dNz;
                    orc_ugimp(ddx, m->dx, m->lpx, &Nx, &dNx);
                    orc_ugimp(ddy, m->dy, m->lpy, &Ny, &dNy);
                    orc_ugimp(ddz, m->dz, m->lpz, &Nz, &dNz);
                    int64_t s = viy - 1;
                    m->Nij[ix + np * s] = Nx * Ny * Nz;
                    m->dNx[ix + np * s] = dNx * Ny * Nz;
                    m->dNy[ix + np * s] = dNy * Nx * Nz;
                    m->dNz[ix + np * s] = dNz * Nx * Ny;
                    m->p2n[ix + np * s] = p2n;
                    viy += 1;
                }
            }
            if (viy > NIC) break;
        }
    }
}

// P2G_OS!, utils_OS.jl:424-452 (2D) and :461-496 (3D)
void orc_p2g(orc_model *m, double G) {
    const int64_t np = m->np, ni = m->ni, NIC = m->nic;
    const bool at = par(m);
#pragma omp parallel for if (at) schedule(static)
    for (int64_t ix = 0; ix < np; ++ix) {
        for (int64_t s = 0; s < NIC; ++s) {
            double Ni = m->Nij[ix + np * s];
            if (Ni == 0.0) continue;
            double dNx = m->dNx[ix + np * s], dNy = m->dNy[ix + np * s];
            int64_t n = m->p2n[ix + np * s] - 1;
            double vol = m->Omega[ix];
            double NiM = m->ms[ix] * Ni;
            atomic_add(&m->g_ms[n], NiM, at);
            if (m->dim == 2) {
                atomic_add(&m->g_ps[n], Ni * m->ps[ix], at);
                atomic_add(&m->g_ps[n + ni], Ni * m->ps[ix + np], at);
                atomic_add(&m->g_fs[n], -vol * (dNx * m->sig[ix] + dNy * m->sig[ix + 3 * np]), at);
                atomic_add(&m->g_fs[n + ni],
                           -vol * (dNy * m->sig[ix + np] + dNx * m->sig[ix + 3 * np]) + NiM * G, at);
            } else {
                double dNz = m->dNz[ix + np * s];
                const double *sg = m->sig;
                atomic_add(&m->g_ps[n], Ni * m->ps[ix], at);
                atomic_add(&m->g_ps[n + ni], Ni * m->ps[ix + np], at);
                atomic_add(&m->g_ps[n + 2 * ni], Ni * m->ps[ix + 2 * np], at);
                atomic_add(&m->g_fs[n],
                           -vol * (dNx * sg[ix] + dNy * sg[ix + 3 * np] + dNz * sg[ix + 5 * np]), at);
                atomic_add(&m->g_fs[n + ni],
                           -vol * (dNy * sg[ix + np] + dNx * sg[ix + 3 * np] + dNz * sg[ix + 4 * np]), at);
                atomic_add(&m->g_fs[n + 2 * ni],
                           -vol * (dNz * sg[ix + 2 * np] + dNx * sg[ix + 5 * np] + dNy * sg[ix + 4 * np]) +
                               NiM * G, at);
            }
        }
    }
}

// solvegrid_a_OS! (va = :a), utils_OS.jl:547-583 / :595-640, and
// solvegrid_OS! (va = :v), utils_OS.jl:507-535 / :650-687
void orc_solvegrid(orc_model *m, double dt) {
    const int64_t ni = m->ni;
    const int D = m->dim;
    const int64_t *idx[3] = {m->vx_idx, m->vy_idx, m->vz_idx};
    const double *val[3] = {m->vx_val, m->vy_val, m->vz_val};
#pragma omp parallel for if (par(m)) schedule(static)
    for (int64_t i = 0; i < ni; ++i) {
        double ms_denom = m->g_ms[i] < mass_eps(m) ? 0.0 : 1.0 / m->g_ms[i];
        if (m->va == ORC_VA_A) {
            for (int d = 0; d < D; ++d)
                if (idx[d][i] != 0) m->g_ps[i + ni * d] = val[d][i];
            for (int d = 0; d < D; ++d) m->g_vs[i + ni * d] = m->g_ps[i + ni * d] * ms_denom;
            double ss = 0.0;
            for (int d = 0; d < D; ++d) ss += m->g_fs[i + ni * d] * m->g_fs[i + ni * d];
            double dampvs = -m->zeta_s * std::sqrt(ss);
            double Fs[3];
            for (int d = 0; d < D; ++d) Fs[d] = m->g_fs[i + ni * d] + dampvs * sgn(m->g_vs[i + ni * d]);
            for (int d = 0; d < D; ++d) m->g_vsT[i + ni * d] = m->g_vs[i + ni * d] + Fs[d] * dt * ms_denom;
            for (int d = 0; d < D; ++d) m->g_as[i + ni * d] = Fs[d] * ms_denom;
            for (int d = 0; d < D; ++d)
                if (idx[d][i] != 0) m->g_vsT[i + ni * d] = val[d][i];
            for (int d = 0; d < D; ++d)
                if (idx[d][i] != 0) m->g_as[i + ni * d] = val[d][i];
            for (int d = 0; d < D; ++d) m->g_ps[i + ni * d] = 0.0;
        } else {
            double P[3];
            for (int d = 0; d < D; ++d) {
                P[d] = m->g_ps[i + ni * d];
                m->g_vs[i + ni * d] = P[d] * ms_denom;
            }
            double ss = 0.0;
            for (int d = 0; d < D; ++d) ss += m->g_fs[i + ni * d] * m->g_fs[i + ni * d];
            double dampvs = -m->zeta_s * std::sqrt(ss);
            for (int d = 0; d < D; ++d) {
                double Fs = m->g_fs[i + ni * d] + dampvs * sgn(m->g_vs[i + ni * d]);
                m->g_vsT[i + ni * d] = (P[d] + Fs * dt) * ms_denom;
            }
            for (int d = 0; d < D; ++d)
                if (idx[d][i] != 0) m->g_vsT[i + ni * d] = val[d][i];
            for (int d = 0; d < D; ++d) m->g_ps[i + ni * d] = 0.0;
        }
    }
}

// solvegrid_a_USL_OS! / solvegrid_USL_OS! (src/solvers/OS_USL.jl:147-320 /
// :24-100): the nodal velocity is advanced in place and the displacement
// increment comes straight from it (no double mapping).  For :a the updated
// velocity is also written to vsT, so that doublemapping1_a_USL_OS! -- which
// maps the updated velocity for both the position and the PIC term -- is the
// MUSL doublemapping1_a_OS! code path of orc_dm1.
void orc_solvegrid_usl(orc_model *m, double dt) {
    const int64_t ni = m->ni;
    const int D = m->dim;
    const int64_t *idx[3] = {m->vx_idx, m->vy_idx, m->vz_idx};
    const double *val[3] = {m->vx_val, m->vy_val, m->vz_val};
#pragma omp parallel for if (par(m)) schedule(static)
    for (int64_t i = 0; i < ni; ++i) {
        double ms_denom = m->g_ms[i] < mass_eps(m) ? 0.0 : 1.0 / m->g_ms[i];
        double ss = 0.0;
        for (int d = 0; d < D; ++d) ss += m->g_fs[i + ni * d] * m->g_fs[i + ni * d];
        const double dampvs = -m->zeta_s * std::sqrt(ss);
        if (m->va == ORC_VA_A) {
            for (int d = 0; d < D; ++d)
                if (idx[d][i] != 0) m->g_ps[i + ni * d] = val[d][i];
            for (int d = 0; d < D; ++d) m->g_vs[i + ni * d] = m->g_ps[i + ni * d] * ms_denom;
            double Fs[3];
            for (int d = 0; d < D; ++d) Fs[d] = m->g_fs[i + ni * d] + dampvs * sgn(m->g_vs[i + ni * d]);
            for (int d = 0; d < D; ++d) m->g_vs[i + ni * d] += Fs[d] * dt * ms_denom;
            for (int d = 0; d < D; ++d) m->g_as[i + ni * d] = Fs[d] * ms_denom;
            for (int d = 0; d < D; ++d)
                if (idx[d][i] != 0) m->g_vs[i + ni * d] = val[d][i];
            for (int d = 0; d < D; ++d)
                if (idx[d][i] != 0) m->g_as[i + ni * d] = val[d][i];
            for (int d = 0; d < D; ++d) {
                m->g_dus[i + ni * d] = m->g_vs[i + ni * d] * dt;
                m->g_vsT[i + ni * d] = m->g_vs[i + ni * d];
            }
        } else {
            for (int d = 0; d < D; ++d) m->g_vs[i + ni * d] = m->g_ps[i + ni * d] * ms_denom;
            for (int d = 0; d < D; ++d) {
                double Fs = m->g_fs[i + ni * d] + dampvs * sgn(m->g_vs[i + ni * d]);
                m->g_vsT[i + ni * d] = (m->g_ps[i + ni * d] + Fs * dt) * ms_denom;
            }
            for (int d = 0; d < D; ++d)
                if (idx[d][i] != 0) m->g_vsT[i + ni * d] = val[d][i];
            for (int d = 0; d < D; ++d) m->g_dus[i + ni * d] = m->g_vsT[i + ni * d] * dt;
        }
    }
}

// doublemapping1_a_OS! (utils_OS.jl:745-788 / :856-908) and
// doublemapping1_OS! (utils_OS.jl:698-743 / :799-854)
void orc_dm1(orc_model *m, double dt) {
    const int64_t np = m->np, ni = m->ni, NIC = m->nic;
    const int D = m->dim;
#pragma omp parallel for if (par(m)) schedule(static)
    for (int64_t ix = 0; ix < np; ++ix) {
        if (m->va == ORC_VA_A) {
            double tv[3] = {0, 0, 0}, tp[3] = {0, 0, 0}, tT[3] = {0, 0, 0};
            for (int64_t s = 0; s < NIC; ++s) {
                double Ni = m->Nij[ix + np * s];
                if (Ni == 0.0) continue;
                int64_t n = m->p2n[ix + np * s] - 1;
                for (int d = 0; d < D; ++d) tp[d] += Ni * m->g_vsT[n + ni * d];
                for (int d = 0; d < D; ++d) tv[d] += Ni * m->g_as[n + ni * d];
                for (int d = 0; d < D; ++d) tT[d] += Ni * m->g_vs[n + ni * d];
            }
            for (int d = 0; d < D; ++d) m->xi[ix + np * d] += tp[d] * dt;
            for (int d = 0; d < D; ++d)
                m->vs[ix + np * d] = m->FLIP * m->vs[ix + np * d] + m->PIC * tT[d] + tv[d] * dt;
            for (int d = 0; d < D; ++d) m->ps[ix + np * d] = m->ms[ix] * m->vs[ix + np * d];
        } else {
            double s1[3] = {0, 0, 0}, s2[3] = {0, 0, 0}, pos[3] = {0, 0, 0};
            for (int64_t s = 0; s < NIC; ++s) {
                double Ni = m->Nij[ix + np * s];
                if (Ni == 0.0) continue;
                int64_t n = m->p2n[ix + np * s] - 1;
                for (int d = 0; d < D; ++d) {
                    double vT = m->g_vsT[n + ni * d];
                    pos[d] += Ni * vT;
                    s1[d] += Ni * (vT - m->g_vs[n + ni * d]);
                    s2[d] += Ni * vT;
                }
            }
            for (int d = 0; d < D; ++d) m->xi[ix + np * d] += dt * pos[d];
            for (int d = 0; d < D; ++d)
                m->vs[ix + np * d] = m->FLIP * (m->vs[ix + np * d] + s1[d]) + m->PIC * s2[d];
            for (int d = 0; d < D; ++d) m->ps[ix + np * d] = m->ms[ix] * m->vs[ix + np * d];
        }
    }
}

// doublemapping2_OS!, utils_OS.jl:917-959
void orc_dm2(orc_model *m) {
    const int64_t np = m->np, ni = m->ni, NIC = m->nic;
    const int D = m->dim;
    const bool at = par(m);
#pragma omp parallel for if (at) schedule(static)
    for (int64_t ix = 0; ix < np; ++ix) {
        for (int64_t s = 0; s < NIC; ++s) {
            double Ni = m->Nij[ix + np * s];
            if (Ni == 0.0) continue;
            int64_t n = m->p2n[ix + np * s] - 1;
            for (int d = 0; d < D; ++d) atomic_add(&m->g_ps[n + ni * d], m->ps[ix + np * d] * Ni, at);
        }
    }
}

// doublemapping3_OS!, utils_OS.jl:968-1016
void orc_dm3(orc_model *m, double dt) {
    const int64_t ni = m->ni;
    const int D = m->dim;
    const int64_t *idx[3] = {m->vx_idx, m->vy_idx, m->vz_idx};
    const double *val[3] = {m->vx_val, m->vy_val, m->vz_val};
#pragma omp parallel for if (par(m)) schedule(static)
    for (int64_t i = 0; i < ni; ++i) {
        double ms_denom = m->g_ms[i] < mass_eps(m) ? 0.0 : 1.0 / m->g_ms[i];
        for (int d = 0; d < D; ++d) m->g_vs[i + ni * d] = m->g_ps[i + ni * d] * ms_denom;
        for (int d = 0; d < D; ++d)
            if (idx[d][i] != 0) m->g_vs[i + ni * d] = val[d][i];
        for (int d = 0; d < D; ++d) m->g_dus[i + ni * d] = m->g_vs[i + ni * d] * dt;
    }
}

// G2P_OS!, utils_OS.jl:1025-1074 (2D) and :1083-1153 (3D)
void orc_g2p(orc_model *m, double dt) {
    const int64_t np = m->np, ni = m->ni, NIC = m->nic;
    const int D = m->dim;
#pragma omp parallel for if (par(m)) schedule(static)
    for (int64_t ix = 0; ix < np; ++ix) {
        double *dF = m->dF, *F = m->F, *de = m->deps, *e = m->eps;
        if (D == 2) {
            double dT1 = 1.0 / dt;
            double dF1 = 0, dF2 = 0, dF3 = 0, dF4 = 0;
            for (int64_t s = 0; s < NIC; ++s) {
                if (m->Nij[ix + np * s] == 0.0) continue;
                int64_t n = m->p2n[ix + np * s] - 1;
                double dNx = m->dNx[ix + np * s], dNy = m->dNy[ix + np * s];
                dF1 += m->g_dus[n] * dNx;
                dF2 += m->g_dus[n] * dNy;
                dF3 += m->g_dus[n + ni] * dNx;
                dF4 += m->g_dus[n + ni] * dNy;
            }
            dF[ix] = dF1; dF[ix + np] = dF2; dF[ix + 2 * np] = dF3; dF[ix + 3 * np] = dF4;
            double exx = dF1 * dT1, eyy = dF4 * dT1, exy = 0.5 * (dF2 + dF3) * dT1;
            m->epsv[ix] = std::sqrt(exx * exx + eyy * eyy + 2.0 * exy * exy);
            de[ix] = dF1; de[ix + np] = dF4; de[ix + 3 * np] = dF2 + dF3;
            e[ix] += dF1; e[ix + np] += dF4; e[ix + 3 * np] += dF2 + dF3;
            double F1 = F[ix], F2 = F[ix + np], F3 = F[ix + 2 * np], F4 = F[ix + 3 * np];
            F[ix] = (dF1 + 1.0) * F1 + dF2 * F3;
            F[ix + np] = (dF1 + 1.0) * F2 + dF2 * F4;
            F[ix + 2 * np] = (dF4 + 1.0) * F3 + dF3 * F1;
            F[ix + 3 * np] = (dF4 + 1.0) * F4 + dF3 * F2;
            double J = F[ix] * F[ix + 3 * np] - F[ix + np] * F[ix + 2 * np];
            m->Omega[ix] = J * m->Omega0[ix];
            m->rho[ix] = m->rho0[ix] / J;
        } else {
            double dT1 = 1.0 / dt;
            double d[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            for (int64_t s = 0; s < NIC; ++s) {
                if (m->Nij[ix + np * s] == 0.0) continue;
                int64_t n = m->p2n[ix + np * s] - 1;
                double dNx = m->dNx[ix + np * s], ds1 = m->g_dus[n];
                double dNy = m->dNy[ix + np * s], ds2 = m->g_dus[n + ni];
                double dNz = m->dNz[ix + np * s], ds3 = m->g_dus[n + 2 * ni];
                d[0] += ds1 * dNx; d[1] += ds1 * dNy; d[2] += ds1 * dNz;
                d[3] += ds2 * dNx; d[4] += ds2 * dNy; d[5] += ds2 * dNz;
                d[6] += ds3 * dNx; d[7] += ds3 * dNy; d[8] += ds3 * dNz;
            }
            for (int k = 0; k < 9; ++k) dF[ix + np * k] = d[k];
            double exx = d[0] * dT1, eyy = d[4] * dT1, ezz = d[8] * dT1;
            double exy = 0.5 * (d[1] + d[3]) * dT1, eyz = 0.5 * (d[5] + d[7]) * dT1,
                   exz = 0.5 * (d[2] + d[6]) * dT1;
            m->epsv[ix] = std::sqrt(exx * exx + eyy * eyy + ezz * ezz +
                                    2.0 * (exy * exy + eyz * eyz + exz * exz));
            de[ix] = d[0]; de[ix + np] = d[4]; de[ix + 2 * np] = d[8];
            de[ix + 3 * np] = d[1] + d[3]; de[ix + 4 * np] = d[5] + d[7]; de[ix + 5 * np] = d[2] + d[6];
            e[ix] += d[0]; e[ix + np] += d[4]; e[ix + 2 * np] += d[8];
            e[ix + 3 * np] += d[1] + d[3]; e[ix + 4 * np] += d[5] + d[7]; e[ix + 5 * np] += d[2] + d[6];
            double f[9];
            for (int k = 0; k < 9; ++k) f[k] = F[ix + np * k];
            double *o = F;
            o[ix] = (d[0] + 1.0) * f[0] + d[1] * f[3] + d[2] * f[6];
            o[ix + np] = (d[0] + 1.0) * f[1] + d[1] * f[4] + d[2] * f[7];
            o[ix + 2 * np] = (d[0] + 1.0) * f[2] + d[1] * f[5] + d[2] * f[8];
            o[ix + 3 * np] = (d[4] + 1.0) * f[3] + d[3] * f[0] + d[5] * f[6];
            o[ix + 4 * np] = (d[4] + 1.0) * f[4] + d[3] * f[1] + d[5] * f[7];
            o[ix + 5 * np] = (d[4] + 1.0) * f[5] + d[3] * f[2] + d[5] * f[8];
            o[ix + 6 * np] = (d[8] + 1.0) * f[6] + d[7] * f[3] + d[6] * f[0];
            o[ix + 7 * np] = (d[8] + 1.0) * f[7] + d[7] * f[4] + d[6] * f[1];
            o[ix + 8 * np] = (d[8] + 1.0) * f[8] + d[7] * f[5] + d[6] * f[2];
            double g[9];
            for (int k = 0; k < 9; ++k) g[k] = F[ix + np * k];
            double J = g[0] * g[4] * g[8] + g[1] * g[5] * g[6] + g[2] * g[3] * g[7] -
                       g[6] * g[4] * g[2] - g[7] * g[5] * g[0] - g[8] * g[3] * g[1];
            m->Omega[ix] = J * m->Omega0[ix];
            m->rho[ix] = m->rho0[ix] / J;
        }
    }
}

// ---------------------------------------------------------------------------
// Two-phase MUSL (procedure!(…, Val(:TS), Val(:MUSL)), src/solvers/TS_MUSL.jl:13-54,
// kernels in src/solvers/utils_TS.jl).  The reference's own path does not run
// as shipped; the restatement keeps its arithmetic and repairs three defects:
//   * submit_work! calls workflow(…, Val(coupling), Val(scheme), Val(va))
//     (src/solver.jl:84-85) but the :TS procedure! takes two Val arguments
//     (TS_MUSL.jl:13-23): here the step is reached whatever va is;
//   * G2P_TS! reads mp.ρs_init / mp.ρw_init (utils_TS.jl:849-850, 953-954), which
//     Particle2D/3D do not have (src/types/particle.jl:60-62 define ρs0 / ρw0),
//     and the 3D kernel writes mp.Δfs (utils_TS.jl:893-895) for ΔFs: the
//     fields meant are used;
//   * resetmpstatus_TS! evaluates the uGIMP basis on the first NIC entries of
//     the 16 / 64 candidate nodes (utils_TS.jl:216-227, 266-283), which leaves
//     support nodes out whenever the particle sits in the right part of its
//     cell: the weights here are the one-phase CPU stencil (support-filtered,
//     resetmpstatus_OS_CPU!, utils_OS.jl:235-277, 363-415).
// Kept as written: grid.mi accumulates N·mw·n (utils_TS.jl:317, 366) while the
// gravity on the mixture uses the particle's mi; iszero (not eps) guards the
// nodal inverses; the 3D G2P_TS! adds the SOLID strain increment to ϵijw
// (utils_TS.jl:929-934; the 2D kernel adds the water increment).
// ---------------------------------------------------------------------------

// resetmpstatus_TS! masses and momenta (utils_TS.jl:205-211, 252-261)
void orc_resetmp_ts(orc_model *m) {
    orc_resetmp(m);   // p2c, weights, ms = Ω·ρs
    const int64_t np = m->np;
    const int D = m->dim;
#pragma omp parallel for if (par(m)) schedule(static)
    for (int64_t ix = 0; ix < np; ++ix) {
        const double n = m->n[ix], vol = m->Omega[ix];
        m->ms[ix] = vol * m->rho[ix];
        m->mw[ix] = vol * m->rhow[ix];
        m->mi[ix] = vol * ((1.0 - n) * m->rho[ix] + n * m->rhow[ix]);
        for (int d = 0; d < D; ++d) {
            m->ps[ix + np * d] = m->ms[ix] * m->vs[ix + np * d] * (1.0 - n);
            m->pw[ix + np * d] = m->mw[ix] * m->vw[ix + np * d] * n;
        }
    }
}

// P2G_TS!, utils_TS.jl:295-334 (2D) and :344-393 (3D)
void orc_p2g_ts(orc_model *m, double G) {
    const int64_t np = m->np, ni = m->ni, NIC = m->nic;
    const int D = m->dim, nv = nv_of(D);
    const bool at = par(m);
#pragma omp parallel for if (at) schedule(static)
    for (int64_t ix = 0; ix < np; ++ix) {
        const double *sg = m->sig;
        double s[6];
        for (int k = 0; k < nv; ++k) s[k] = sg[ix + np * k];
        const double n = m->n[ix], sw = m->sigw[ix], vol = m->Omega[ix];
        const double tdg = (n * m->mw[ix] * G) / m->kperm[m->nid[ix] - 1];
        for (int64_t q = 0; q < NIC; ++q) {
            const double Ni = m->Nij[ix + np * q];
            if (Ni == 0.0) continue;
            const double dN[3] = {m->dNx[ix + np * q], m->dNy[ix + np * q], D == 3 ? m->dNz[ix + np * q] : 0.0};
            const int64_t nd = m->p2n[ix + np * q] - 1;
            atomic_add(&m->g_ms[nd], Ni * m->ms[ix] * (1.0 - n), at);
            atomic_add(&m->g_mi[nd], Ni * m->mw[ix] * n, at);
            atomic_add(&m->g_mw[nd], Ni * m->mw[ix], at);
            for (int d = 0; d < D; ++d) {
                atomic_add(&m->g_ps[nd + ni * d], Ni * m->ps[ix + np * d], at);
                atomic_add(&m->g_pw[nd + ni * d], Ni * m->pw[ix + np * d], at);
            }
            // water force: −Ω ∂N σw (+ N mw G on the last axis)
            for (int d = 0; d < D; ++d) {
                double f = -vol * (dN[d] * sw);
                if (d == D - 1) f += Ni * m->mw[ix] * G;
                atomic_add(&m->g_fw[nd + ni * d], f, at);
            }
            // mixture force: −Ω (∂N (σ + σw I)) (+ N mi G on the last axis)
            double fs[3];
            if (D == 2) {
                fs[0] = -vol * (dN[0] * (s[0] + sw) + dN[1] * s[3]);
                fs[1] = -vol * (dN[1] * (s[1] + sw) + dN[0] * s[3]) + Ni * m->mi[ix] * G;
            } else {
                fs[0] = -vol * (dN[0] * (s[0] + sw) + dN[1] * s[3] + dN[2] * s[5]);
                fs[1] = -vol * (dN[1] * (s[1] + sw) + dN[0] * s[3] + dN[2] * s[4]);
                fs[2] = -vol * (dN[2] * (s[2] + sw) + dN[0] * s[5] + dN[1] * s[4]) + Ni * m->mi[ix] * G;
            }
            for (int d = 0; d < D; ++d) {
                atomic_add(&m->g_fs[nd + ni * d], fs[d], at);
                atomic_add(&m->g_fd[nd + ni * d], Ni * tdg * (m->vw[ix + np * d] - m->vs[ix + np * d]), at);
            }
        }
    }
}

// solvegrid_TS!, utils_TS.jl:404-455 (2D) and :465-532 (3D)
void orc_solvegrid_ts(orc_model *m, double dt) {
    const int64_t ni = m->ni;
    const int D = m->dim;
    const int64_t *si[3] = {m->vx_idx, m->vy_idx, m->vz_idx}, *wi[3] = {m->vxw_idx, m->vyw_idx, m->vzw_idx};
    const double *sv[3] = {m->vx_val, m->vy_val, m->vz_val}, *wv[3] = {m->vxw_val, m->vyw_val, m->vzw_val};
#pragma omp parallel for if (par(m)) schedule(static)
    for (int64_t i = 0; i < ni; ++i) {
        const double msd = m->g_ms[i] == 0.0 ? 0.0 : 1.0 / m->g_ms[i];
        const double mwd = m->g_mw[i] == 0.0 ? 0.0 : 1.0 / m->g_mw[i];
        double vs[3], vw[3], fs[3], fw[3];
        for (int d = 0; d < D; ++d) {
            vs[d] = m->g_ps[i + ni * d] * msd;
            vw[d] = m->g_pw[i + ni * d] * mwd;
            fs[d] = m->g_fs[i + ni * d];
            fw[d] = m->g_fw[i + ni * d];
            m->g_vs[i + ni * d] = vs[d];
            m->g_vw[i + ni * d] = vw[d];
        }
        double qw = 0.0, qs = 0.0;
        for (int d = 0; d < D; ++d) {
            qw += fw[d] * fw[d];
            qs += (fs[d] - fw[d]) * (fs[d] - fw[d]);
        }
        const double tw = -m->zeta_w * std::sqrt(qw), ts_ = -m->zeta_s * std::sqrt(qs);
        for (int d = 0; d < D; ++d) {
            const double dw = tw * sgn(vw[d]), ds = ts_ * sgn(vs[d]);
            const double aw = mwd * (fw[d] + dw + m->g_fd[i + ni * d]);
            const double as = msd * (-m->g_mi[i] * aw + fs[d] + dw + ds);
            m->g_aw[i + ni * d] = aw;
            m->g_as[i + ni * d] = as;
            m->g_vsT[i + ni * d] = vs[d] + as * dt;
            m->g_vwT[i + ni * d] = vw[d] + aw * dt;
        }
        for (int d = 0; d < D; ++d) {
            if (si[d][i] != 0) m->g_vsT[i + ni * d] = sv[d][i];
            if (wi[d][i] != 0) m->g_vwT[i + ni * d] = wv[d][i];
        }
        for (int d = 0; d < D; ++d) {
            m->g_ps[i + ni * d] = 0.0;
            m->g_pw[i + ni * d] = 0.0;
        }
    }
}

// doublemapping1_TS!, utils_TS.jl:543-585 (2D) and :596-648 (3D)
void orc_dm1_ts(orc_model *m, double dt) {
    const int64_t np = m->np, ni = m->ni, NIC = m->nic;
    const int D = m->dim;
#pragma omp parallel for if (par(m)) schedule(static)
    for (int64_t ix = 0; ix < np; ++ix) {
        double pos[3] = {0, 0, 0}, s1[3] = {0, 0, 0}, s2[3] = {0, 0, 0}, w1[3] = {0, 0, 0}, w2[3] = {0, 0, 0};
        for (int64_t q = 0; q < NIC; ++q) {
            const double Ni = m->Nij[ix + np * q];
            if (Ni == 0.0) continue;
            const int64_t nd = m->p2n[ix + np * q] - 1;
            for (int d = 0; d < D; ++d) {
                const double vT = m->g_vsT[nd + ni * d], wT = m->g_vwT[nd + ni * d];
                pos[d] += Ni * vT;
                s1[d] += Ni * (vT - m->g_vs[nd + ni * d]);
                s2[d] += Ni * vT;
                w1[d] += Ni * (wT - m->g_vw[nd + ni * d]);
                w2[d] += Ni * wT;
            }
        }
        const double n = m->n[ix];
        for (int d = 0; d < D; ++d) {
            m->xi[ix + np * d] += dt * pos[d];
            m->vs[ix + np * d] = m->FLIP * (m->vs[ix + np * d] + s1[d]) + m->PIC * s2[d];
            m->vw[ix + np * d] = m->FLIP * (m->vw[ix + np * d] + w1[d]) + m->PIC * w2[d];
            m->ps[ix + np * d] = m->ms[ix] * m->vs[ix + np * d] * (1.0 - n);
            m->pw[ix + np * d] = m->mw[ix] * m->vw[ix + np * d] * n;
        }
    }
}

// doublemapping2_TS!, utils_TS.jl:657-704
void orc_dm2_ts(orc_model *m) {
    const int64_t np = m->np, ni = m->ni, NIC = m->nic;
    const int D = m->dim;
    const bool at = par(m);
#pragma omp parallel for if (at) schedule(static)
    for (int64_t ix = 0; ix < np; ++ix) {
        for (int64_t q = 0; q < NIC; ++q) {
            const double Ni = m->Nij[ix + np * q];
            if (Ni == 0.0) continue;
            const int64_t nd = m->p2n[ix + np * q] - 1;
            for (int d = 0; d < D; ++d) {
                atomic_add(&m->g_ps[nd + ni * d], m->ps[ix + np * d] * Ni, at);
                atomic_add(&m->g_pw[nd + ni * d], m->pw[ix + np * d] * Ni, at);
            }
        }
    }
}

// doublemapping3_TS!, utils_TS.jl:713-780
void orc_dm3_ts(orc_model *m, double dt) {
    const int64_t ni = m->ni;
    const int D = m->dim;
    const int64_t *si[3] = {m->vx_idx, m->vy_idx, m->vz_idx}, *wi[3] = {m->vxw_idx, m->vyw_idx, m->vzw_idx};
    const double *sv[3] = {m->vx_val, m->vy_val, m->vz_val}, *wv[3] = {m->vxw_val, m->vyw_val, m->vzw_val};
#pragma omp parallel for if (par(m)) schedule(static)
    for (int64_t i = 0; i < ni; ++i) {
        const double msd = m->g_ms[i] == 0.0 ? 0.0 : 1.0 / m->g_ms[i];
        const double mwd = m->g_mw[i] == 0.0 ? 0.0 : 1.0 / m->g_mw[i];
        for (int d = 0; d < D; ++d) {
            double vs = m->g_ps[i + ni * d] * msd, vw = m->g_pw[i + ni * d] * mwd;
            if (si[d][i] != 0) vs = sv[d][i];
            if (wi[d][i] != 0) vw = wv[d][i];
            m->g_vs[i + ni * d] = vs;
            m->g_vw[i + ni * d] = vw;
            m->g_dus[i + ni * d] = vs * dt;
            m->g_duw[i + ni * d] = vw * dt;
        }
    }
}

// G2P_TS!, utils_TS.jl:790-857 (2D) and :867-961 (3D): the solid part is
// G2P_OS!'s arithmetic (same expressions), then the water strain, the pore
// pressure and the porosity.
void orc_g2p_ts(orc_model *m, double dt) {
    const int64_t np = m->np, ni = m->ni, NIC = m->nic;
    const int D = m->dim, nv = nv_of(D);
    std::vector<double> vol_old(m->Omega, m->Omega + np);
    orc_g2p(m, dt);   // ΔFs, ϵv, Δϵijs, ϵijs, F, J, Ω, ρs = ρs0 / J
#pragma omp parallel for if (par(m)) schedule(static)
    for (int64_t ix = 0; ix < np; ++ix) {
        double dw[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int64_t q = 0; q < NIC; ++q) {
            if (m->Nij[ix + np * q] == 0.0) continue;
            const int64_t nd = m->p2n[ix + np * q] - 1;
            const double dN[3] = {m->dNx[ix + np * q], m->dNy[ix + np * q], D == 3 ? m->dNz[ix + np * q] : 0.0};
            for (int a = 0; a < D; ++a)
                for (int b = 0; b < D; ++b) dw[a * D + b] += m->g_duw[nd + ni * a] * dN[b];
        }
        const double *dF = m->dF;
        double *ew = m->epsw, *dew = m->depsw;
        double trs, trw;
        if (D == 2) {
            dew[ix] = dw[0]; dew[ix + np] = dw[3]; dew[ix + 3 * np] = dw[1] + dw[2];
            ew[ix] += dw[0]; ew[ix + np] += dw[3]; ew[ix + 3 * np] += dw[1] + dw[2];
            trs = dF[ix] + dF[ix + 3 * np];
            trw = dw[0] + dw[3];
        } else {
            dew[ix] = dw[0]; dew[ix + np] = dw[4]; dew[ix + 2 * np] = dw[8];
            dew[ix + 3 * np] = dw[1] + dw[3]; dew[ix + 4 * np] = dw[5] + dw[7]; dew[ix + 5 * np] = dw[2] + dw[6];
            const double d0 = dF[ix], d1 = dF[ix + np], d2 = dF[ix + 2 * np], d3 = dF[ix + 3 * np],
                         d4 = dF[ix + 4 * np], d5 = dF[ix + 5 * np], d6 = dF[ix + 6 * np],
                         d7 = dF[ix + 7 * np], d8 = dF[ix + 8 * np];
            ew[ix] += d0; ew[ix + np] += d4; ew[ix + 2 * np] += d8;   // solid increments, as written
            ew[ix + 3 * np] += d1 + d3; ew[ix + 4 * np] += d5 + d7; ew[ix + 5 * np] += d2 + d6;
            trs = d0 + d4 + d8;
            trw = dw[0] + dw[4] + dw[8];
        }
        (void)nv;
        double J;
        const double *F = m->F;
        if (D == 2) {
            J = F[ix] * F[ix + 3 * np] - F[ix + np] * F[ix + 2 * np];
        } else {
            double g[9];
            for (int k = 0; k < 9; ++k) g[k] = F[ix + np * k];
            J = g[0] * g[4] * g[8] + g[1] * g[5] * g[6] + g[2] * g[3] * g[7] - g[6] * g[4] * g[2] -
                g[7] * g[5] * g[0] - g[8] * g[3] * g[1];
        }
        const double dJ = J * m->Omega0[ix] / vol_old[ix];
        m->rhow[ix] = m->rhow0[ix] / J;
        const double n = m->n[ix];
        m->sigw[ix] += (m->Kw[m->nid[ix] - 1] / n) * ((1.0 - n) * trs + n * trw);
        m->n[ix] = 1.0 - (1.0 - n) / dJ;
    }
}

}  // extern "C"

namespace {

// liE!, src/materials/linearelastic.jl:22-69 (2D) and :78-140 (3D).
// s points at sig[ix + np*k] columns; works on a local copy.
void liE_point(int D, double *s, const double *dF, const double *de, double Ks, double Gt,
               double *sm, double *sij, double *s_rot) {
    if (D == 2) {
        double w = 0.5 * (dF[1] - dF[2]);
        double s1 = s[0], s2 = s[1], s4 = s[3];
        s[0] += w * s4 * 2.0;
        s[1] += -w * s4 * 2.0;
        s[3] += w * (s2 - s1);
    } else {
        double wxy = 0.5 * (dF[3] - dF[1]);
        double wyz = 0.5 * (dF[7] - dF[5]);
        double wxz = 0.5 * (dF[6] - dF[2]);
        double s1 = s[0], s2 = s[1], s3 = s[2], s4 = s[3], s5 = s[4], s6 = s[5];
        s[0] += 2.0 * (s4 * wxy + s6 * wxz);
        s[1] += -2.0 * (s4 * wxy - s5 * wyz);
        s[2] += -2.0 * (s6 * wxz + s5 * wyz);
        s[3] += wxy * (s2 - s1) + wxz * s5 + wyz * s6;
        s[4] += wyz * (s3 - s2) - wxz * s4 - wxy * s6;
        s[5] += wxz * (s3 - s1) + wxy * s5 - wyz * s4;
    }
    if (s_rot) for (int k = 0; k < (D == 2 ? 4 : 6); ++k) s_rot[k] = s[k];
    double Dt = Ks + 1.333333 * Gt;
    double Dd = Ks - 0.666667 * Gt;
    s[0] += Dt * de[0] + Dd * de[1] + Dd * de[2];
    s[1] += Dd * de[0] + Dt * de[1] + Dd * de[2];
    s[2] += Dd * de[0] + Dd * de[1] + Dt * de[2];
    s[3] += Gt * de[3];
    if (D == 3) { s[4] += Gt * de[4]; s[5] += Gt * de[5]; }
    double m = (s[0] + s[1] + s[2]) * 0.333333;
    *sm = m;
    sij[0] = s[0] - m; sij[1] = s[1] - m; sij[2] = s[2] - m; sij[3] = s[3];
    if (D == 3) { sij[4] = s[4]; sij[5] = s[5]; }
}

// dpP!, src/materials/druckerprager.jl:22-80 (2D) and :89-155 (3D)
void dp_point(int D, double *s, double *sm, double *sij, double *epsq, double *epsk,
              double K, double G, double c, double phi, double psi, double sigt) {
    double m = *sm;
    double tau;
    if (D == 2)
        tau = std::sqrt(0.5 * (sij[0] * sij[0] + sij[1] * sij[1] + sij[2] * sij[2]) + sij[3] * sij[3]);
    else
        tau = std::sqrt(0.5 * (sij[0] * sij[0] + sij[1] * sij[1] + sij[2] * sij[2]) + sij[3] * sij[3] +
                        sij[4] * sij[4] + sij[5] * sij[5]);
    double kphi = (6.0 * c * std::cos(phi)) / (1.732051 * (3.0 + std::sin(phi)));
    double qphi = (6.0 * std::sin(phi)) / (1.732051 * (3.0 + std::sin(phi)));
    double qpsi = (6.0 * std::sin(psi)) / (1.732051 * (3.0 + std::sin(psi)));
    double st = std::min(sigt, kphi / qphi);
    double ab = std::sqrt(1.0 + qphi * qphi) - qphi;
    double tb = kphi - qphi * st;
    double fs = tau + qphi * m - kphi;
    double ft = m - st;
    double BF = (tau - tb) - (ab * (m - st));
    const int nv = D == 2 ? 4 : 6;
    if (((m < st) && (fs > 0.0)) || ((m >= st) && (BF > 0.0))) {
        double dl = fs / (G + K * qphi * qpsi);
        double t1 = m - K * qpsi * dl;
        double t2 = (kphi - qphi * t1) / tau;
        s[0] = sij[0] * t2 + t1;
        s[1] = sij[1] * t2 + t1;
        s[2] = sij[2] * t2 + t1;
        for (int k = 3; k < nv; ++k) s[k] = sij[k] * t2;
        *epsq += dl * std::sqrt(0.333333 + 0.222222 * qpsi * qpsi);
        *epsk += dl * qpsi;
    }
    if ((m >= st) && (BF <= 0.0)) {
        double dl = ft / K;
        s[0] = sij[0] + st;
        s[1] = sij[1] + st;
        s[2] = sij[2] + st;
        *epsq += dl * 0.333333 * 1.414214;
        *epsk += dl;
    }
    double mm = (s[0] + s[1] + s[2]) * 0.333333;
    *sm = mm;
    sij[0] = s[0] - mm; sij[1] = s[1] - mm; sij[2] = s[2] - mm;
    for (int k = 3; k < nv; ++k) sij[k] = s[k];
}

// mcP! 2D, src/materials/mohrcoulomb.jl:22-86
void mc2d_point(double *s, double *sm, double *sij, double *epsq, double *epsk, double K,
                double G, double c0, double Hp, double cr, double phi) {
    double c = std::max(c0 + Hp * (*epsq), cr);
    double ds = s[0] - s[1];
    double tau = std::sqrt(0.25 * ds * ds + s[3] * s[3]);
    double sig = 0.5 * (s[0] + s[1]);
    double f = tau + sig * std::sin(phi) - c * std::cos(phi);
    double sn1 = s[0], sn2 = s[1], sn3 = s[2], sn4 = s[3];
    double beta = std::fabs(c * std::cos(phi) - sig * std::sin(phi)) / tau;
    double dsigA = 0.5 * beta * ds;
    double dsigB = c / std::tan(phi);
    if ((sig <= dsigB) && (f > 0.0)) {
        sn1 = sig + dsigA;
        sn2 = sig - dsigA;
        sn4 = beta * s[3];
    }
    if ((sig > dsigB) && (f > 0.0)) {
        sn1 = dsigB;
        sn2 = dsigB;
        sn4 = 0.0;
    }
    double d1 = sn1 - s[0], d2 = sn2 - s[1], d3 = sn3 - s[2], d4 = sn4 - s[3];
    s[0] = sn1; s[1] = sn2; s[2] = sn3; s[3] = sn4;
    double Dt = K + 1.333333 * G;
    double Dd = K - 0.666667 * G;
    double base = 1.0 / ((Dd - Dt) * (2.0 * Dd + Dt));
    double exx = -(Dd * d1 + Dt * d1 - Dd * d2 - Dd * d3) * base;
    double eyy = -(-Dd * d1 + Dd * d2 + Dt * d2 - Dd * d3) * base;
    double ezz = -(-Dd * d1 - Dd * d2 + Dd * d3 + Dt * d3) * base;
    double exy = d4 / G;
    *epsk = exx + eyy + ezz;
    *epsq += std::sqrt(0.666667 * (exx * exx + eyy * eyy + ezz * ezz + exy * exy * 2.0));
    double mm = (s[0] + s[1] + s[2]) * 0.333333;
    *sm = mm;
    sij[0] = s[0] - mm; sij[1] = s[1] - mm; sij[2] = s[2] - mm; sij[3] = s[3];
}

}  // namespace

extern "C" {

void orc_dp_point(int dim, double *sig, double *epsq, double *epsk, double K, double G, double c,
                  double phi, double psi, double sigt) {
    double sij[6], sm = (sig[0] + sig[1] + sig[2]) * 0.333333;
    for (int k = 0; k < (dim == 2 ? 4 : 6); ++k) sij[k] = k < 3 ? sig[k] - sm : sig[k];
    dp_point(dim, sig, &sm, sij, epsq, epsk, K, G, c, phi, psi, sigt);
}

// liE! then dpP!/mcP! (OS_MUSL.jl:82-96), per particle.  The 3D mcP! body is
// commented out in the reference (mohrcoulomb.jl:152-455): literal mode keeps
// the elastic predictor; restated mode applies orc_mc3d_point.
void orc_constitutive(orc_model *m, double Ti) {
    const int64_t np = m->np;
    const int D = m->dim, nv = nv_of(D), nd = D * D;
#pragma omp parallel for if (par(m)) schedule(static)
    for (int64_t ix = 0; ix < np; ++ix) {
        int64_t mat = m->nid[ix] - 1;
        double s[6], dF[9], de[6], sij[6], sm;
        for (int k = 0; k < nv; ++k) { s[k] = m->sig[ix + np * k]; de[k] = m->deps[ix + np * k]; }
        for (int k = 0; k < nd; ++k) dF[k] = m->dF[ix + np * k];
        double srot[6];
        liE_point(D, s, dF, de, m->Ks[mat], m->Gs[mat], &sm, sij, srot);
        if (Ti >= m->Te) {
            if (m->constitutive == ORC_DRUCKERPRAGER) {
                dp_point(D, s, &sm, sij, &m->epsq[ix], &m->epsk[ix], m->Ks[mat], m->Gs[mat], m->c[mat],
                         m->phi[mat], m->psi[mat], m->sigt[mat]);
            } else if (m->constitutive == ORC_MOHRCOULOMB) {
                if (D == 2) {
                    mc2d_point(s, &sm, sij, &m->epsq[ix], &m->epsk[ix], m->Ks[mat], m->Gs[mat], m->c[mat],
                               m->Hp[mat], m->cr[mat], m->phi[mat]);
                } else if (m->mc3d == ORC_MC3D_RESTATED) {
                    orc_mc3d_point(s, srot, de, &m->epsq[ix], m->Ks[mat], m->Gs[mat], m->c[mat],
                                   m->phi[mat], m->psi[mat], m->sigt[mat]);
                    sm = (s[0] + s[1] + s[2]) * 0.333333;
                    for (int k = 0; k < 6; ++k) sij[k] = k < 3 ? s[k] - sm : s[k];
                }
            }
        }
        for (int k = 0; k < nv; ++k) { m->sig[ix + np * k] = s[k]; m->sij[ix + np * k] = sij[k]; }
        m->sigm[ix] = sm;
    }
}

// vollock1_OS! / vollock2_OS!, utils_OS.jl:1162-1257
static void orc_vollock(orc_model *m) {
    const int64_t np = m->np;
    const int nv = nv_of(m->dim);
    for (int64_t ix = 0; ix < np; ++ix) {
        int64_t c = m->p2c[ix] - 1;
        double vol = m->Omega[ix];
        m->g_sigm[c] += vol * m->sigm[ix];
        m->g_omega[c] += vol;
    }
    for (int64_t ix = 0; ix < np; ++ix) {
        int64_t c = m->p2c[ix] - 1;
        double sm = m->g_sigm[c] / m->g_omega[c];
        double *s = m->sig, *sij = m->sij;
        s[ix] = sij[ix] + sm;
        s[ix + np] = sij[ix + np] + sm;
        s[ix + 2 * np] = sij[ix + 2 * np] + sm;
        for (int k = 3; k < nv; ++k) s[ix + np * k] = sij[ix + np * k];
        double mm = (s[ix] + s[ix + np] + s[ix + 2 * np]) * 0.333333;
        m->sigm[ix] = mm;
        sij[ix] = s[ix] - mm; sij[ix + np] = s[ix + np] - mm; sij[ix + 2 * np] = s[ix + 2 * np] - mm;
        for (int k = 3; k < nv; ++k) sij[ix + np * k] = s[ix + np * k];
    }
}

// procedure!(…, Val(:OS), Val(:MUSL), Val(:a|:v)), src/solvers/OS_MUSL.jl:12-102
int orc_procedure(orc_model *m, double dt, double Ti) {
#ifdef _OPENMP
    if (m->nthreads > 1) omp_set_num_threads(m->nthreads);
#endif
    double G = Ti < m->Te ? m->gravity / m->Te * Ti : m->gravity;
    orc_resetgrid(m);
    if (m->coupling == 1) {   // procedure!(…, Val(:TS), Val(:MUSL)), TS_MUSL.jl:24-53
        orc_resetmp_ts(m);
        orc_p2g_ts(m, G);
        orc_solvegrid_ts(m, dt);
        orc_dm1_ts(m, dt);
        orc_dm2_ts(m);
        orc_dm3_ts(m, dt);
        orc_g2p_ts(m, dt);
        orc_constitutive(m, Ti);
        return 0;
    }
    orc_resetmp(m);
    orc_p2g(m, G);
    if (m->scheme == 1) {   // USL, src/solvers/OS_USL.jl:102-145, 325-368
        orc_solvegrid_usl(m, dt);
        orc_dm1(m, dt);
    } else {
        orc_solvegrid(m, dt);
        orc_dm1(m, dt);
        orc_dm2(m);
        orc_dm3(m, dt);
    }
    orc_g2p(m, dt);
    orc_constitutive(m, Ti);
    if (m->mvl) orc_vollock(m);
    return 0;
}

// The host time loop of submit_work!, src/solver.jl:118-125 (Ti += ΔT in FP64).
int orc_run(orc_model *m, double dt, double Ti0, int64_t nsteps, double *Ti_out) {
    double Ti = Ti0;
    for (int64_t k = 0; k < nsteps; ++k) {
        int rc = orc_procedure(m, dt, Ti);
        if (rc) return rc;
        Ti += dt;
    }
    if (Ti_out) *Ti_out = Ti;
    return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Restated 3D Mohr-Coulomb return mapping.
//
// The reference's 3D mcP! body is commented out (mohrcoulomb.jl:152-455), so the
// reference's own 3D result is the elastic predictor only (literal mode).  This
// restatement follows the predictor-corrector structure of
// src/materials/mohr_coulomb.tcc:3-138 (trial state, yield state, lambda from the
// trial and from the pre-increment stress, up to 100 corrections with tolerance
// 0.1) with the invariants, yield functions and derivatives written out in the
// commented Julia (mohrcoulomb.jl:108-126 invariants, :203-221 yield functions,
// :223-331 dF/dsigma, :332-407 dP/dsigma).  Deliberate choices where the
// commented Julia is incomplete: classification threshold 0 (a state is
// "yielding" when its yield function is > 0); non-tensile states use the shear
// derivatives; no softening (dphi/dpstrain = dc/dpstrain = 0).
// Voigt order xx, yy, zz, xy, yz, zx with engineering shear strains.
// ---------------------------------------------------------------------------
namespace {

struct MCInv { double sm, j2, j3, rho, theta, epsilon; double dev[6]; };

void mc_invariants(const double *s, MCInv *v) {
    double sm = (s[0] + s[1] + s[2]) / 3.0;
    v->sm = sm;
    double d0 = s[0] - sm, d1 = s[1] - sm, d2 = s[2] - sm;
    v->dev[0] = d0; v->dev[1] = d1; v->dev[2] = d2; v->dev[3] = s[3]; v->dev[4] = s[4]; v->dev[5] = s[5];
    double j2 = ((s[0] - s[1]) * (s[0] - s[1]) + (s[1] - s[2]) * (s[1] - s[2]) +
                 (s[2] - s[0]) * (s[2] - s[0])) / 6.0 + s[3] * s[3] + s[4] * s[4] + s[5] * s[5];
    double j3 = d0 * d1 * d2 + 2.0 * s[3] * s[4] * s[5] - d0 * s[4] * s[4] - d1 * s[5] * s[5] -
                d2 * s[3] * s[3];
    double lv = std::fabs(j2) > DBL_EPSILON ? (3.0 * std::sqrt(3.0) / 2.0) * (j3 / std::pow(j2, 1.5)) : 0.0;
    lv = std::min(1.0, std::max(-1.0, lv));
    v->j2 = j2; v->j3 = j3;
    v->theta = std::acos(lv) / 3.0;
    v->rho = std::sqrt(2.0 * j2);
    v->epsilon = std::sqrt(3.0) * sm;
}

enum { MC_ELASTIC = 0, MC_TENSILE = 1, MC_SHEAR = 2 };

int mc_yield(const MCInv &v, double phi, double c, double st, double *ft, double *fs) {
    const double r23 = std::sqrt(2.0 / 3.0), r15 = std::sqrt(1.5), r3 = std::sqrt(3.0);
    *ft = r23 * std::cos(v.theta) * v.rho + v.epsilon / r3 - st;
    *fs = r15 * v.rho * (std::sin(v.theta + M_PI / 3.0) / (r3 * std::cos(phi)) +
                         std::cos(v.theta + M_PI / 3.0) * std::tan(phi) / 3.0) +
          (v.epsilon / r3) * std::tan(phi) - c;
    int type = MC_ELASTIC;
    if (*ft > 0.0 && *fs > 0.0) {
        double nphi = (1.0 + std::sin(phi)) / (1.0 - std::sin(phi));
        double sp = st * nphi - 2.0 * c * std::sqrt(nphi);
        double ap = std::sqrt(1.0 + nphi * nphi) + nphi;
        double h = *ft + ap * (r23 * std::cos(v.theta - 4.0 * M_PI / 3.0) * v.rho + v.epsilon / r3 - sp);
        type = h > DBL_EPSILON ? MC_TENSILE : MC_SHEAR;
    } else if (*fs > 0.0) {
        type = MC_SHEAR;
    } else if (*ft > 0.0) {
        type = MC_TENSILE;
    }
    return type;
}

void mc_df_dp(int type, const MCInv &v, double phi, double psi, double c, double st,
              double *df, double *dp, double *dp_dq) {
    const double r23 = std::sqrt(2.0 / 3.0), r15 = std::sqrt(1.5), r3 = std::sqrt(3.0);
    const double th = v.theta, rho = v.rho;
    double df_de, df_dr, df_dt;
    if (type == MC_TENSILE) {
        df_de = 1.0 / r3;
        df_dr = r23 * std::cos(th);
        df_dt = -r23 * rho * std::sin(th);
    } else {
        df_de = std::tan(phi) / r3;
        df_dr = r15 * (std::sin(th + M_PI / 3.0) / (r3 * std::cos(phi)) +
                       std::cos(th + M_PI / 3.0) * std::tan(phi) / 3.0);
        df_dt = r15 * rho * (std::cos(th + M_PI / 3.0) / (r3 * std::cos(phi)) -
                             std::sin(th + M_PI / 3.0) * std::tan(phi) / 3.0);
    }
    double de_ds[6] = {1.0 / r3, 1.0 / r3, 1.0 / r3, 0, 0, 0};
    double dr_ds[6] = {0, 0, 0, 0, 0, 0};
    if (rho > DBL_EPSILON)
        for (int k = 0; k < 6; ++k) dr_ds[k] = (k < 3 ? v.dev[k] : 2.0 * v.dev[k]) / rho;
    const double *d = v.dev;
    double dj2[6] = {d[0], d[1], d[2], 2.0 * d[3], 2.0 * d[4], 2.0 * d[5]};
    // rows of the deviatoric tensor (xx, xy, zx), (xy, yy, yz), (zx, yz, zz)
    double r1[3] = {d[0], d[3], d[5]}, r2[3] = {d[3], d[1], d[4]}, r3v[3] = {d[5], d[4], d[2]};
    double dj3[6];
    dj3[0] = r1[0] * r1[0] + r1[1] * r1[1] + r1[2] * r1[2] - 2.0 / 3.0 * v.j2;
    dj3[1] = r2[0] * r2[0] + r2[1] * r2[1] + r2[2] * r2[2] - 2.0 / 3.0 * v.j2;
    dj3[2] = r3v[0] * r3v[0] + r3v[1] * r3v[1] + r3v[2] * r3v[2] - 2.0 / 3.0 * v.j2;
    dj3[3] = 2.0 * (r1[0] * r2[0] + r1[1] * r2[1] + r1[2] * r2[2]);
    dj3[4] = 2.0 * (r2[0] * r3v[0] + r2[1] * r3v[1] + r2[2] * r3v[2]);
    dj3[5] = 2.0 * (r1[0] * r3v[0] + r1[1] * r3v[1] + r1[2] * r3v[2]);
    double dr_dj2 = -9.0 * std::sqrt(3.0) / 4.0 * v.j3, dr_dj3 = 3.0 * std::sqrt(3.0) / 2.0;
    double dt_dr = -1.0 / 3.0;
    if (std::fabs(v.j2) > DBL_EPSILON) {
        double r = v.j3 * 0.5 * std::pow(v.j2 / 3.0, -1.5);
        dr_dj2 *= std::pow(v.j2, -2.5);
        dr_dj3 *= std::pow(v.j2, -1.5);
        double fac = std::fabs(1.0 - r * r) < DBL_EPSILON ? DBL_EPSILON : std::fabs(1.0 - r * r);
        dt_dr = -1.0 / (3.0 * std::sqrt(fac));
    }
    double dt_ds[6];
    for (int k = 0; k < 6; ++k) dt_ds[k] = dt_dr * (dr_dj2 * dj2[k] + dr_dj3 * dj3[k]);
    for (int k = 0; k < 6; ++k) df[k] = df_de * de_ds[k] + df_dr * dr_ds[k] + df_dt * dt_ds[k];
    const double ct = std::cos(th), sn = std::sin(th);
    double dp_de, dp_dr, dp_dt;
    if (type == MC_TENSILE) {
        const double et = 0.6, xit = 0.1;
        double sq = 4.0 * (1.0 - et * et) * ct * ct + 5.0 * et * et - 4.0 * et;
        if (sq < DBL_EPSILON) sq = 0.00001;
        double rt_den = 2.0 * (1.0 - et * et) * ct + (2.0 * et - 1.0) * std::sqrt(sq);
        double rt_num = 4.0 * (1.0 - et * et) * ct * ct + (2.0 * et - 1.0) * (2.0 * et - 1.0);
        if (rt_den < DBL_EPSILON) rt_den = 0.00001;
        double rt = rt_num / (3.0 * rt_den);
        double den = std::sqrt(xit * xit * st * st + 1.5 * rt * rt * rho * rho);
        double dp_drt = 1.5 * rho * rho * rt / den;
        dp_dr = 1.5 * rho * rt * rt / den;
        dp_de = 1.0 / r3;
        double drtden_dt = -2.0 * (1.0 - et * et) * sn -
                           (2.0 * et - 1.0) * 4.0 * (1.0 - et * et) * ct * sn / std::sqrt(sq);
        double drtnum_dt = -8.0 * (1.0 - et * et) * ct * sn;
        double drt_dt = (drtnum_dt * rt_den - drtden_dt * rt_num) / (3.0 * rt_den * rt_den);
        dp_dt = dp_drt * drt_dt;
    } else {
        double rmc = (3.0 - std::sin(phi)) / (6.0 * std::cos(phi));
        double e = (3.0 - std::sin(phi)) / (3.0 + std::sin(phi));
        if (e <= 0.5) e = 0.5000000001;
        else if (e > 1.0) e = 1.0;
        double sq = 4.0 * (1.0 - e * e) * ct * ct + 5.0 * e * e - 4.0 * e;
        if (sq < DBL_EPSILON) sq = 0.00001;
        double mm = 2.0 * (1.0 - e * e) * ct + (2.0 * e - 1.0) * std::sqrt(sq);
        if (mm < DBL_EPSILON) mm = 0.00001;
        double l = 4.0 * (1.0 - e * e) * ct * ct + (2.0 * e - 1.0) * (2.0 * e - 1.0);
        double rmw = (l / mm) * rmc;
        const double xi = 0.1;
        double om = (xi * c * std::tan(psi)) * (xi * c * std::tan(psi)) + (rmw * r15 * rho) * (rmw * r15 * rho);
        if (om < DBL_EPSILON) om = 0.00001;
        double dl_dt = -8.0 * (1.0 - e * e) * ct * sn;
        double dm_dt = -2.0 * (1.0 - e * e) * sn + 0.5 * (2.0 * e - 1.0) * dl_dt / std::sqrt(sq);
        double drmw_dt = (mm * dl_dt - l * dm_dt) / (mm * mm);
        dp_de = std::tan(psi) / r3;
        dp_dr = 3.0 * rho * rmw * rmw / (2.0 * std::sqrt(om));
        dp_dt = 3.0 * rho * rho * rmw * rmc * drmw_dt / (2.0 * std::sqrt(om));
    }
    for (int k = 0; k < 6; ++k) dp[k] = dp_de * de_ds[k] + dp_dr * dr_ds[k] + dp_dt * dt_ds[k];
    *dp_dq = dp_dr * r23;
}

// y = De x for the isotropic elastic matrix (engineering shear).
inline void De_mul(double K, double G, const double *x, double *y) {
    double Dt = K + 4.0 / 3.0 * G, Dd = K - 2.0 / 3.0 * G;
    y[0] = Dt * x[0] + Dd * x[1] + Dd * x[2];
    y[1] = Dd * x[0] + Dt * x[1] + Dd * x[2];
    y[2] = Dd * x[0] + Dd * x[1] + Dt * x[2];
    y[3] = G * x[3]; y[4] = G * x[4]; y[5] = G * x[5];
}

inline double dot6(const double *a, const double *b) {
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2] + a[3] * b[3] + a[4] * b[4] + a[5] * b[5];
}

}  // namespace

// the restated 3D Mohr-Coulomb yield functions (tension ft, shear fs) of a stress;
// returns the state (0 elastic, 1 tensile, 2 shear)
extern "C" int orc_mc3d_yield(const double *sig, double c, double phi, double st, double *ft, double *fs) {
    MCInv v;
    mc_invariants(sig, &v);
    return mc_yield(v, phi, c, st, ft, fs);
}

extern "C" void orc_mc3d_point(double *sig, const double *sig0, const double *de, double *epsq,
                               double K, double G, double c, double phi, double psi, double st) {
    const double tol = 1e-1;
    MCInv v;
    double ft, fs, df[6], dp[6], dq, Ddp[6], Ddf[6];
    mc_invariants(sig, &v);
    int type_tr = mc_yield(v, phi, c, st, &ft, &fs);
    if (type_tr == MC_ELASTIC) return;
    mc_df_dp(type_tr, v, phi, psi, c, st, df, dp, &dq);
    De_mul(K, G, df, Ddf);   // De symmetric: (df^T De) = (De df)^T
    double y_tr = type_tr == MC_TENSILE ? ft : fs;
    double lam_tr = y_tr / dot6(Ddf, dp);
    double dp_tr[6], dq_tr = dq;
    for (int k = 0; k < 6; ++k) dp_tr[k] = dp[k];
    // lambda from the pre-increment stress
    MCInv v0;
    double ft0, fs0, df0[6], dp0[6], dq0, Ddf0[6];
    mc_invariants(sig0, &v0);
    int type0 = mc_yield(v0, phi, c, st, &ft0, &fs0);
    double y0 = type0 == MC_TENSILE ? ft0 : (type0 == MC_SHEAR ? fs0 : DBL_MAX);
    mc_df_dp(type0, v0, phi, psi, c, st, df0, dp0, &dq0);
    De_mul(K, G, df0, Ddf0);
    double lam0 = dot6(Ddf0, de) / dot6(Ddf0, dp0);
    double upd[6];
    for (int k = 0; k < 6; ++k) upd[k] = sig[k];
    double dpd;
    if (std::fabs(y0) < tol) {
        De_mul(K, G, dp0, Ddp);
        for (int k = 0; k < 6; ++k) upd[k] -= lam0 * Ddp[k];
        dpd = lam0 * dq0;
    } else {
        De_mul(K, G, dp_tr, Ddp);
        for (int k = 0; k < 6; ++k) upd[k] -= lam_tr * Ddp[k];
        dpd = lam_tr * dq_tr;
    }
    for (int it = 0; it < 100; ++it) {
        mc_invariants(upd, &v);
        int t = mc_yield(v, phi, c, st, &ft, &fs);
        if (ft < tol && fs < tol) break;
        mc_df_dp(t, v, phi, psi, c, st, df, dp, &dq);
        De_mul(K, G, df, Ddf);
        double y = t == MC_TENSILE ? ft : fs;
        double lam = y / dot6(Ddf, dp);
        De_mul(K, G, dp, Ddp);
        for (int k = 0; k < 6; ++k) upd[k] -= lam * Ddp[k];
        dpd += lam * dq;
    }
    for (int k = 0; k < 6; ++k) sig[k] = upd[k];
    *epsq += dpd;
}
