/*
 * mpm_oracle.h -- FP64 CPU restatement of MaterialPointSolver.jl's one-phase
 * uGIMP step (TEST INFRASTRUCTURE ONLY: used by tests/, bench.py's CPU baseline
 * and __graft_entry__.smoke() as the checker; never linked into the product).
 *
 * Parity status: UNPINNED by the reference.  The reference is pure Julia, Julia
 * is not installed, and the reference's own tests hold no golden vectors for
 * this path (test/runtests.jl is `@test 1==1`).  This restatement is
 * cross-checked against hand-derived known-answer tests and against an
 * independent pure-Python transliteration (tests/oracle_py.py).
 *
 * All arrays use the reference's memory layout: Julia column-major `n x k`
 * matrices, i.e. component k of item i lives at a[i + n*k]; indices stored in
 * the arrays (p2c, p2n, nid, bc idx) are 1-based like the reference's.
 */
#ifndef MPM_ORACLE_H
#define MPM_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_LINEARELASTIC = 0, ORC_DRUCKERPRAGER = 1, ORC_MOHRCOULOMB = 2 };
enum { ORC_VA_A = 0, ORC_VA_V = 1 };
enum { ORC_MC3D_LITERAL = 0, ORC_MC3D_RESTATED = 1 };

typedef struct {
    /* ---- grid (Grid2D / Grid3D, src/types/grid.jl) ---- */
    int32_t dim;                /* 2 or 3 */
    int32_t nic;                /* NIC: 9 (2D) or 27 (3D) */
    int64_t nnx, nny, nnz;      /* nnz = 1 in 2D */
    int64_t ncx, ncy, ncz;      /* ncz = 1 in 2D */
    int64_t ni, nc;
    double x1, y1, z1, dx, dy, dz;
    const double *g_xi;         /* ni x dim node coordinates (grid.ξ) */
    double *g_ms;               /* ni */
    double *g_ps, *g_fs, *g_vs, *g_vsT, *g_as, *g_dus; /* ni x dim */
    double *g_sigm, *g_omega;   /* nc (cell mean stress / volume, MVL) */
    /* ---- particles (Particle2D / Particle3D, src/types/particle.jl) ---- */
    int64_t np;
    double lpx, lpy, lpz;       /* mp.dx, mp.dy, mp.dz */
    int64_t *p2c;               /* np */
    int64_t *p2n;               /* np x NIC */
    double *Nij, *dNx, *dNy, *dNz; /* np x NIC */
    double *xi;                 /* np x dim */
    double *vs, *ps;            /* np x dim */
    double *ms, *Omega, *Omega0, *rho, *rho0; /* np */
    double *sig, *eps, *deps, *sij; /* np x nv (nv = 4 in 2D, 6 in 3D) */
    double *sigm, *epsq, *epsk, *epsv; /* np */
    double *dF, *F;             /* np x dim^2 */
    /* ---- property (Property, src/types/property.jl) ---- */
    const int64_t *nid;         /* np, 1-based material id */
    const double *Ks, *Gs, *c, *phi, *psi, *sigt, *Hp, *cr; /* per material */
    /* ---- velocity boundary (VBoundary2D/3D, src/types/boundary.jl) ---- */
    const int64_t *vx_idx, *vy_idx, *vz_idx; /* ni */
    const double *vx_val, *vy_val, *vz_val;  /* ni */
    /* ---- args (Args2D/3D, src/types/modelargs.jl) ---- */
    double Te, gravity, FLIP, PIC, zeta_s;
    int32_t constitutive, va, mvl, mc3d;
    int32_t nthreads;           /* 0/1: sequential literal order; >1: OpenMP */
    int32_t scheme;             /* 0: MUSL (OS_MUSL.jl), 1: USL (OS_USL.jl) */
    /* ---- two-phase coupling (:TS, src/solvers/TS_MUSL.jl, utils_TS.jl) ---- */
    int32_t coupling;           /* 0: :OS, 1: :TS */
    int32_t f32;                /* 1: the reference's float type T2 is Float32 (massless-node cutoff eps(T2)) */
    double zeta_w;              /* ζw */
    double *g_mi, *g_mw;        /* ni */
    double *g_pw, *g_fw, *g_fd, *g_vw, *g_vwT, *g_aw, *g_duw; /* ni x dim */
    double *mw, *mi, *n, *rhow, *rhow0, *sigw; /* np */
    double *vw, *pw;            /* np x dim */
    double *epsw, *depsw;       /* np x nv */
    const double *Kw, *kperm;   /* per material: water bulk modulus, permeability k */
    const int64_t *vxw_idx, *vyw_idx, *vzw_idx; /* ni: water velocity BC */
    const double *vxw_val, *vyw_val, *vzw_val;
} orc_model;

/* One call of procedure!(…, Val(:OS), Val(:MUSL), Val(va)), src/solvers/OS_MUSL.jl:12-102 */
int orc_procedure(orc_model *m, double dt, double Ti);
/* nsteps calls with Ti accumulated like src/solver.jl:118-125 (FP64). */
int orc_run(orc_model *m, double dt, double Ti0, int64_t nsteps, double *Ti_out);

/* Individual stages, for per-stage parity tests. */
void orc_resetgrid(orc_model *m);
void orc_resetmp(orc_model *m);
void orc_p2g(orc_model *m, double G);
void orc_solvegrid(orc_model *m, double dt);
void orc_solvegrid_usl(orc_model *m, double dt);
void orc_dm1(orc_model *m, double dt);
void orc_dm2(orc_model *m);
void orc_dm3(orc_model *m, double dt);
void orc_g2p(orc_model *m, double dt);
void orc_constitutive(orc_model *m, double Ti);
/* Two-phase stages (utils_TS.jl); orc_procedure runs them when coupling = 1. */
void orc_resetmp_ts(orc_model *m);
void orc_p2g_ts(orc_model *m, double G);
void orc_solvegrid_ts(orc_model *m, double dt);
void orc_dm1_ts(orc_model *m, double dt);
void orc_dm2_ts(orc_model *m);
void orc_dm3_ts(orc_model *m, double dt);
void orc_g2p_ts(orc_model *m, double dt);

/* Julia float fld/cld and the p2c formula (utils_OS.jl:247-249, 380-383). */
double orc_fld(double a, double b);
double orc_cld(double a, double b);
void orc_p2c(const orc_model *m, const double *xi, int64_t np, int64_t *p2c_out);
/* 1-D uGIMP basis, src/toolkits/mpbasisfunc.jl:40-53 (CPU division form). */
void orc_ugimp(double d, double h, double lp, double *N, double *dN);
/* Single-particle return mappings (for known-answer tests).  sig/sij in/out, nv comps. */
void orc_dp_point(int dim, double *sig, double *epsq, double *epsk,
                  double K, double G, double c, double phi, double psi, double sigt);
/* Restated 3D Mohr-Coulomb: sig = elastic trial (in/out), sig0 = rotated
 * pre-increment stress, de = strain increment (engineering shear). */
/* Restated 3D Mohr-Coulomb yield functions of a stress (Voigt); returns 0 elastic, 1 tensile, 2 shear. */
int orc_mc3d_yield(const double *sig, double c, double phi, double st, double *ft, double *fs);
void orc_mc3d_point(double *sig, const double *sig0, const double *de, double *epsq,
                    double K, double G, double c, double phi, double psi, double sigt);

#ifdef __cplusplus
}
#endif
#endif
