/*
 * mpm_b200.h -- C ABI of libmpm_b200.so, the B200 (sm_100a) backend for the
 * one-phase explicit uGIMP MPM step of MaterialPointSolver.jl.
 *
 * The entry points replace the reference's device boundary and step workflow
 * (paths relative to the MaterialPointSolver.jl repository):
 *
 *   mpm_create + mpm_upload   host2device   ext/CUDAExt/devicehelpfunc_cuda.jl:17-37
 *   mpm_step                  procedure!    src/solvers/OS_MUSL.jl:12-102, called
 *                                           per step by submit_work!, src/solver.jl:84,119
 *   mpm_download              device2host!  ext/CUDAExt/devicehelpfunc_cuda.jl:39-69
 *   mpm_destroy               clean_device! ext/CUDAExt/devicehelpfunc_cuda.jl:71-100
 *   mpm_compute_p2c           the p2c part of resetmpstatus_OS!, src/solvers/utils_OS.jl:203-205,325-328
 *   mpm_peak_bandwidth        Tpeak,        ext/CUDAExt/devicehelpfunc_cuda.jl:102-136
 *   mpm_snapshot, mpm_h5_*    the HDF5 snapshots of submit_work!, src/solver.jl:54-111
 *
 * Host arrays are passed as views of the caller's arrays in the reference's
 * layout: Julia column-major `n x k` matrices (component k of item i at
 * ptr[i + ld*k]), element type tagged per view, indices 1-based.
 *
 * Conventions: every function returns MPM_OK (0) or a negative MPM_E_* code;
 * nothing throws across the ABI; mpm_last_error() returns the message of the
 * last failure on a handle.  One handle is used by one host thread at a time.
 * All device memory belongs to the handle until mpm_destroy().
 */
#ifndef MPM_B200_H
#define MPM_B200_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MPM_ABI_VERSION 1

/* return codes */
#define MPM_OK 0
#define MPM_E_ARG (-1)           /* invalid argument / descriptor */
#define MPM_E_CUDA (-2)          /* CUDA runtime error (message has details) */
#define MPM_E_OUT_OF_GRID (-3)   /* a particle's stencil left the grid */
#define MPM_E_NONPOSITIVE_J (-4) /* det(F) <= 0 on some particle */
#define MPM_E_NAN (-5)           /* non-finite particle state */
#define MPM_E_STATE (-6)         /* call out of order (e.g. step before upload) */
#define MPM_E_CELL_OVERFLOW (-7) /* more particles in one cell than the sort handles */
#define MPM_E_UNSUPPORTED (-8)   /* option not provided by this backend */

/* constitutive models (Args.constitutive) */
#define MPM_LINEARELASTIC 0
#define MPM_DRUCKERPRAGER 1
#define MPM_MOHRCOULOMB 2

/* arithmetic of the device step */
#define MPM_PREC_MIXED 0 /* FP32 bulk, FP64 positions and det(F)/volume */
#define MPM_PREC_FP64 1  /* all FP64 (self-check mode) */

/* velocity update mode (Args.va) */
#define MPM_VA_A 0
#define MPM_VA_V 1

/* update scheme (args.scheme) */
#define MPM_SCHEME_MUSL 0
#define MPM_SCHEME_USL 1
/* coupling: one-phase (OS_*.jl) or two-phase solid + water (TS_MUSL.jl, MUSL only;
 * restated: the reference's own two-phase path does not run as shipped) */
#define MPM_COUPLING_OS 0
#define MPM_COUPLING_TS 1

/* 3D Mohr-Coulomb: the reference's 3D mcP! body is commented out, so its 3D
 * "mohrcoulomb" run is the elastic predictor only (LITERAL).  RESTATED applies
 * the predictor-corrector Mohr-Coulomb return mapping. */
#define MPM_MC3D_LITERAL 0
#define MPM_MC3D_RESTATED 1

/* element type tags of host views */
#define MPM_T_F64 0
#define MPM_T_F32 1
#define MPM_T_I64 2
#define MPM_T_I32 3

typedef struct mpm_handle mpm_handle;

/* Model description: grid (Grid2D/3D), particle sizes (Particle2D/3D dx,dy,dz)
 * and run arguments (Args2D/3D). */
typedef struct {
    int32_t abi_version;   /* MPM_ABI_VERSION */
    int32_t dim;           /* 2 or 3 */
    int32_t precision;     /* MPM_PREC_* */
    int32_t device;        /* CUDA device ordinal */
    int64_t np;            /* particles (mp.np) */
    int64_t nmat;          /* materials (length of the Property arrays) */
    int64_t nnx, nny, nnz; /* nodes per axis (grid.nnx, nny, nnz; nnz = 1 in 2D) */
    double x1, y1, z1;     /* grid origin */
    double dx, dy, dz;     /* cell size */
    double lpx, lpy, lpz;  /* particle size (mp.dx, mp.dy, mp.dz) */
    int32_t constitutive;  /* MPM_LINEARELASTIC / DRUCKERPRAGER / MOHRCOULOMB */
    int32_t va;            /* MPM_VA_A / MPM_VA_V */
    int32_t mvl;           /* Args.MVL */
    int32_t mc3d;          /* MPM_MC3D_* */
    double FLIP, PIC;      /* Args.FLIP, Args.PIC */
    double zeta_s;         /* Args.ζs */
    double gravity;        /* Args.gravity */
    double Te;             /* Args.Te */
    int32_t time_f32;      /* 1: accumulate Ti in Float32 (reference FP32 mode) */
    int32_t sort_every;    /* re-sort period in steps (0 = library default) */
    int32_t scheme;        /* MPM_SCHEME_MUSL (OS_MUSL.jl) or MPM_SCHEME_USL (OS_USL.jl) */
    int32_t coupling;      /* MPM_COUPLING_OS or MPM_COUPLING_TS (Args.coupling) */
    double zeta_w;         /* Args.ζw (two-phase water damping) */
} mpm_desc;

/* A host array view. */
typedef struct {
    void *ptr;     /* NULL = not supplied */
    int32_t type;  /* MPM_T_* */
    int32_t pad;
    int64_t ld;    /* leading dimension (rows) of the column-major array */
} mpm_view;

/* Host views of the reference structs' arrays (names as in the reference). */
typedef struct {
    /* Particle2D/3D */
    mpm_view xi;      /* ξ      np x dim   */
    mpm_view vs;      /* vs     np x dim   */
    mpm_view sig;     /* σij    np x 4|6   (Voigt xx,yy,zz,xy[,yz,zx]) */
    mpm_view eps;     /* ϵijs   np x 4|6   */
    mpm_view epsq;    /* ϵq     np         */
    mpm_view epsk;    /* ϵk     np         */
    mpm_view epsv;    /* ϵv     np         */
    mpm_view Omega;   /* Ω      np         */
    mpm_view Omega0;  /* Ω0     np         */
    mpm_view rho;     /* ρs     np         */
    mpm_view rho0;    /* ρs0    np         */
    mpm_view F;       /* F      np x dim^2 (row-major components) */
    mpm_view ms;      /* ms     np         (download only) */
    mpm_view sigm;    /* σm     np         (download only) */
    mpm_view p2c;     /* p2c    np         (download only, 1-based) */
    /* Property */
    mpm_view nid;     /* nid    np         (1-based material id) */
    mpm_view Ks, Gs, c, phi, psi, sigt, Hp, cr; /* nmat each */
    /* VBoundary2D/3D, per node in the reference's node order */
    mpm_view vx_idx, vx_val, vy_idx, vy_val, vz_idx, vz_val;
    /* two-phase (coupling = TS): Particle2D/3D water fields, Property Kw and k,
     * VBoundary water velocity BC (vx_w_idx … vz_w_val; absent = none) */
    mpm_view n;       /* n      np         porosity */
    mpm_view rhow;    /* ρw     np         (upload; download: ρw0 / J) */
    mpm_view sigw;    /* σw     np         pore pressure */
    mpm_view vw;      /* vw     np x dim   */
    mpm_view epsw;    /* ϵijw   np x 4|6   */
    mpm_view mw;      /* mw     np         (download only) */
    mpm_view Kw, kperm; /* nmat each */
    mpm_view vxw_idx, vxw_val, vyw_idx, vyw_val, vzw_idx, vzw_val;
} mpm_host_views;

/* download field mask */
#define MPM_F_XI (1u << 0)
#define MPM_F_VS (1u << 1)
#define MPM_F_SIG (1u << 2)
#define MPM_F_EPS (1u << 3)
#define MPM_F_EPSQ (1u << 4)
#define MPM_F_EPSK (1u << 5)
#define MPM_F_EPSV (1u << 6)
#define MPM_F_OMEGA (1u << 7)
#define MPM_F_MS (1u << 8)
#define MPM_F_SIGM (1u << 9)
#define MPM_F_F (1u << 10)
#define MPM_F_RHO (1u << 11)
#define MPM_F_P2C (1u << 12)
#define MPM_F_MW (1u << 13)     /* two-phase fields */
#define MPM_F_VW (1u << 14)
#define MPM_F_SIGW (1u << 15)
#define MPM_F_EPSW (1u << 16)
#define MPM_F_N (1u << 17)
#define MPM_F_RHOW (1u << 18)
/* the set device2host! copies (devicehelpfunc_cuda.jl:46-55) */
#define MPM_F_REFERENCE (MPM_F_SIGM | MPM_F_VS | MPM_F_XI | MPM_F_OMEGA | MPM_F_SIG | \
                         MPM_F_EPSK | MPM_F_EPSQ | MPM_F_EPSV | MPM_F_EPS | MPM_F_MS)
/* ... and the two-phase additions (devicehelpfunc_cuda.jl:56-62) */
#define MPM_F_REFERENCE_TS (MPM_F_REFERENCE | MPM_F_MW | MPM_F_VW | MPM_F_SIGW | MPM_F_EPSW | MPM_F_N)

typedef struct {
    int64_t steps_done;        /* steps run on this handle */
    int64_t sorts_done;        /* particle re-sorts */
    int64_t active_nodes;      /* nodes with mass > 0 in the current P2G accumulators */
    int64_t launches;          /* kernel launches issued by this handle so far */
    int32_t error_flags;       /* sticky device error bits (MPM_E_* as 1 << -code) */
    int32_t kernels_per_step;  /* kernel launches per step */
    double last_step_ms;       /* device time of the last mpm_step call, ms */
    double device_bytes;       /* device memory held by the handle, bytes */
    int64_t surr_rows;         /* returns handed to the surrogate so far */
    int64_t surr_fallbacks;    /* of those, returns redone by the plain return */
} mpm_stats;

/* ---- lifecycle (host2device / clean_device!) ---- */
int mpm_create(const mpm_desc *desc, mpm_handle **out);
/* mpm_upload / mpm_download: the host arrays may be pageable or page-locked;
 * both calls return once every copy into or out of them has completed (with
 * page-locked arrays the copies run asynchronously inside the call and the
 * host-side conversions overlap them).  Staging uses the model's own particle
 * buffers, no device allocation. */
int mpm_upload(mpm_handle *h, const mpm_host_views *v);
int mpm_destroy(mpm_handle *h);

/* ---- the step (procedure!) ----
 * Runs `nsteps` consecutive steps starting at time Ti0 with step dt; Ti is
 * advanced like submit_work!'s `Ti += ΔT` (in Float32 if desc.time_f32).
 * Returns after the device finished; *Ti_out (optional) receives the end time. */
int mpm_step(mpm_handle *h, double dt, double Ti0, int64_t nsteps, double *Ti_out);
/* Asynchronous variant on the handle's stream; errors surface at mpm_sync. */
int mpm_step_async(mpm_handle *h, double dt, double Ti0, int64_t nsteps);
int mpm_sync(mpm_handle *h);

/* ---- tuning (no counterpart in the reference) ----
 * Run-time choices of the step: the cell re-sort period (steps), the
 * particle-pass variant (0 = per-particle kernels whose scatters merge the
 * windows of neighbouring lanes and reduce into L2, the default; 1 =
 * shared-memory tiled kernels; 2 = box passes: one warp per tile of 32 cells
 * with the tile's node data in shared memory, in FP32 with va = :a and no
 * PIC/MVL/USL/two-phase, else variant 0; 3 = variant 0 with the fused pass
 * compiled for 3 instead of 4 resident CTAs per SM, i.e. 85 instead of 64
 * registers, for the FP32 one-phase MUSL step without the restated 3D
 * Mohr-Coulomb, else variant 0; variant 3 is the default of 3D models, variant
 * 0 of 2D ones) and the sort's tile shape (cells; 3D 2x8x2
 * (default), 4x8x1, 4x4x2; 2D 4x8 (default), 2x16; mpm_set_tile re-sorts at
 * the next step).  mpm_autotune times, on REAL steps of the model (they advance
 * the simulation exactly like mpm_step, from Ti0, and *Ti_out receives the end
 * time), every tile shape with the re-sort periods 8, 16, 32, 64 (default
 * passes), then variant 3 at the best shape so far with periods 32 and 64,
 * then the tiled and the box passes at periods 16 and 32; each trial runs
 * max(steps_per_trial, period) steps starting with a sort.  Since the trials
 * advance the model (and a growing flow makes later trials slower), the
 * fastest variant-0 candidate and the fastest other candidate are then timed
 * again back to back, 64 steps each, and the faster of the two is kept
 * (mpm_get_tile reports its shape).  Each timed run's ms per step goes to
 * trial_ms (optional, trial_cap entries) in that order, the two final runs
 * last. */
int mpm_set_tuning(mpm_handle *h, int32_t sort_every, int32_t tiled);
int mpm_get_tuning(mpm_handle *h, int32_t *sort_every, int32_t *tiled);
int mpm_set_tile(mpm_handle *h, int32_t tx, int32_t ty, int32_t tz);
int mpm_get_tile(mpm_handle *h, int32_t *tx, int32_t *ty, int32_t *tz);
int mpm_autotune(mpm_handle *h, double dt, double Ti0, int64_t steps_per_trial, double *Ti_out,
                 int32_t *sort_every_out, int32_t *tiled_out, double *trial_ms, int32_t trial_cap);

/* ---- results (device2host!) ---- */
int mpm_download(mpm_handle *h, const mpm_host_views *v, uint32_t field_mask);
/* p2c (1-based, the reference's formula) of the current positions, original order. */
int mpm_compute_p2c(mpm_handle *h, int64_t *p2c_out);
/* Current device order: out[k] = 0-based original index of the k-th stored particle. */
int mpm_download_order(mpm_handle *h, int64_t *order_out);
/* Re-sort particles by cell now (normally done every desc.sort_every steps). */
int mpm_sort(mpm_handle *h);

/* ---- grid introspection for per-stage checks ----
 * Runs the stages of one step selected by stage_mask (bit 0 P2G, 1 grid solve,
 * 2 double mapping (DM1+DM2), 3 DM3, 4 G2P + stress) at time Ti, then copies
 * grid field `field` (0 mass, 1 momentum, 2 force, 3 vsT, 4 as, 5 Δu, 6 vs)
 * into host (ni x dim column-major FP64, reference node order). */
int mpm_run_stages(mpm_handle *h, double dt, double Ti, uint32_t stage_mask);
int mpm_download_grid(mpm_handle *h, int32_t field, double *out);

/* ---- cell ordering without allocation ----
 * No counterpart in the reference (which never reorders particles).  For
 * callers that cannot allocate device memory -- a host runtime that owns all
 * device memory through its own pool, a real-time loop that must not hit the
 * allocator's implicit synchronisation -- this computes what mpm_compute_p2c() and mpm_sort() +
 * mpm_download_order() compute for particles in their original order:
 * p2c_out[i] (1-based, the reference's formula) and order_out[k] (0-based
 * index of the k-th particle in the library's cell-sorted order).  All five
 * pointers are caller-owned DEVICE buffers (x, y, z: np FP64 coordinates; z is
 * unused in 2D; order_out, p2c_out: np int64).  The grid and np come from
 * `d` (the other descriptor fields are ignored).  The work runs on `stream`
 * (a cudaStream_t; NULL = the legacy default stream) and the call is
 * synchronous: it copies an error word back and waits for the stream before
 * returning, so it must not be called on a stream that is being captured, and
 * should get a non-blocking stream while another thread captures a graph.
 *
 * The scratch is a fixed static device array of MPM_NOALLOC_SCRATCH_BYTES
 * that every GPU loading the library holds until process exit; np above
 * MPM_NOALLOC_MAX_PARTICLES or a grid above MPM_NOALLOC_MAX_KEYS cell keys
 * (cells rounded up to whole 2x8x2 / 4x8 tiles) is rejected with MPM_E_ARG.
 * The first call on each device looks up the scratch's device address (with
 * that device current); make it before any stream capture.  All calls share
 * the one scratch array, so calls whose work overlaps on the GPU race: issue
 * them on one stream or serialise them.  Errors: mpm_last_error(NULL). */
#define MPM_NOALLOC_MAX_PARTICLES (1 << 19)
#define MPM_NOALLOC_MAX_KEYS (1 << 19)
#define MPM_NOALLOC_SCRATCH_BYTES 14780416
int mpm_cell_order_noalloc(const mpm_desc *d, const double *x, const double *y, const double *z,
                           int64_t *order_out, int64_t *p2c_out, void *stream);

/* ---- random fields (grf_gc! / grf_ec!, src/toolkits/randomfield.jl:57-96, 112-150) ----
 * Evaluates the randomised-spectral sum of those functions on the device, FP64:
 *   out[i] = scale * sum_j ( a_j sin(V_j . p_i) + b_j cos(V_j . p_i) ),
 * p_i = (x[i], y[i], z[i]) (z may be NULL: 0), harm = nh rows of
 * (V1, V2, V3, a, b), row-major.  The caller draws the harmonics (the
 * reference's rand/randn loop) and applies the final rescaling.  x, y, z,
 * harm and out are HOST arrays; the call is synchronous.  Errors:
 * mpm_last_error(NULL). */
int mpm_grf_eval(int32_t device, const double *x, const double *y, const double *z, int64_t np,
                 const double *harm, int64_t nh, double scale, double *out);

/* ---- stress-return surrogate (no counterpart in the reference) ----
 * A 15 -> 64 -> 64 -> 64 -> 6 MLP (GELU in the tanh form of Hendrycks & Gimpel
 * 2016, hardware tanh) standing in for the Drucker-Prager /
 * Mohr-Coulomb return (druckerprager.jl:89-155), BF16 weights and FP32
 * accumulation on the tensor cores (tcgen05).  params: mpm_mlp_nparams() FP32
 * master values, per layer W[k][n] then b[n] with the input padded to 16 and
 * the output to 16 (padding stays zero).  norm: 64 floats, input mean[16],
 * input std[16], output mean[16], output std[16].  feat: n x 16 FP32 (15
 * features + 1 pad), target / out: n x 6.  All arrays are DEVICE pointers, the
 * work is queued on `stream` (a cudaStream_t, NULL = default); err (device int)
 * gets bit 0 set if a tensor-core completion wait timed out. */
int mpm_mlp_nparams(void);
#define MPM_MLP_RESIDUAL 1   /* flags: the network predicts out - feat[0..5] (the correction) */
/* flags, test hook of the tensor-core completion wait: issue no MMA and wait
 * with a short limit, so the wait times out, *err gets bit 0 and no output is
 * written; the context stays usable (nothing is in flight when the CTA leaves) */
#define MPM_MLP_TEST_STALL 2
int mpm_mlp_forward(const float *params, const float *norm, const float *feat, float *out, int64_t n,
                    int32_t flags, int *err, void *stream);
/* Adds the gradient of 1/2 * inv_btot * sum (MLP(x) - y)^2 (normalised units)
 * over the n samples to grad, and that loss to *loss. */
int mpm_mlp_grad(const float *params, const float *norm, const float *feat, const float *target, int64_t n,
                 float inv_btot, int32_t flags, float *grad, float *loss, int *err, void *stream);
/* One Adam step (bias correction for step count `step` >= 1); zeroes grad. */
int mpm_mlp_adam(float *params, float *grad, float *m, float *v, float lr, float b1, float b2, float eps,
                 int64_t step, void *stream);

/* The surrogate inside the step (3D Drucker-Prager, or the restated 3D
 * Mohr-Coulomb return of desc.mc3d = MPM_MC3D_RESTATED): with on = 1 every
 * yielding particle's return is deferred, the MLP (params / norm: HOST arrays
 * as above, copied) predicts it, and the prediction is kept when its yield
 * residual is at most tol -- Drucker-Prager: |f| / max(kphi, |qphi sigma_m|,
 * sref); Mohr-Coulomb: the yield function of the trial's mode at the
 * prediction, and neither yield function above it, relative to max(c,
 * |sigma_m| tan(phi), sref) -- else the plain return (dpP! / the restated
 * Mohr-Coulomb predictor-corrector) is used.  Drucker-Prager plastic strains
 * follow the plain return's closed-form multiplier; an accepted Mohr-Coulomb
 * row adds the plastic shear strain of its stress correction to epsq.
 * Counts in mpm_stats.surr_rows / surr_fallbacks.  on = 0 restores the plain
 * return. */
int mpm_set_surrogate(mpm_handle *h, const float *params, const float *norm, int32_t flags, float tol, float sref,
                      int32_t on);
/* Training samples from plain steps (3D Drucker-Prager or restated
 * Mohr-Coulomb): one yielding particle in `every` (hashed
 * by index and step) writes its 16 features (trial stress 6, strain increment
 * 6, plastic strain, cohesion, friction, 0) to feat and the plain return's
 * stress to target (DEVICE arrays of cap rows); *count (device) counts rows
 * offered, rows beyond cap are dropped.  every = 0 stops logging. */
int mpm_log_samples(mpm_handle *h, float *feat, float *target, uint32_t *count, uint32_t cap, uint32_t every);

/* ---- snapshots (the HDF5 output of submit_work!, src/solver.jl:54-111) ----
 * mpm_h5 is an HDF5 file written by the library itself (no libhdf5): groups of
 * contiguous datasets, readable by HDF5.jl / h5py.  mpm_h5_write stores one
 * dataset `name` ("group3/stress"; missing groups are created) of `rank`
 * dimensions given slowest-varying first: HDF5.jl writes a Julia np x k
 * matrix as dims {k, np}, so its column-major buffer is passed that way; rank
 * 0 is a scalar.  The file becomes readable when mpm_h5_close returns.  Calls
 * on one file are serialised internally.  Errors: mpm_last_error(NULL).
 *
 * mpm_snapshot enqueues one group of submit_work! (src/solver.jl:60-70):
 * "group<group>/" + stress, strain_s, eqstrain, ekstrain, eqrate, coords,
 * velocity_s, volume, mass_s (the fields of field_mask, a subset of
 * MPM_F_SNAPSHOT; two-phase models also pressure_w, strain_w, velocity_w,
 * porosity, MPM_F_SNAPSHOT_TS) in the original particle order, and "time" = Ti, all of
 * element type `type` (MPM_T_F64 or MPM_T_F32).  It returns at once: the
 * fields are gathered on the handle's stream behind the steps issued so far,
 * copied to pinned host memory on a second stream while later steps run, and
 * written by a writer thread.  Two snapshots can be in flight; a third call
 * waits for the older one.  mpm_snapshot_wait returns when every enqueued
 * snapshot is in the file (written = groups written so far) and reports a
 * writer error once; call it before mpm_h5_close. */
typedef struct mpm_h5 mpm_h5;
int mpm_h5_create(const char *path, mpm_h5 **out);
int mpm_h5_write(mpm_h5 *f, const char *name, int32_t type, int32_t rank, const int64_t *dims,
                 const void *data);
int mpm_h5_close(mpm_h5 *f);
#define MPM_F_SNAPSHOT (MPM_F_SIG | MPM_F_EPS | MPM_F_EPSQ | MPM_F_EPSK | MPM_F_EPSV | MPM_F_XI | \
                        MPM_F_VS | MPM_F_OMEGA | MPM_F_MS)
/* two-phase groups add pressure_w, strain_w, velocity_w, porosity (src/solver.jl:73-76) */
#define MPM_F_SNAPSHOT_TS (MPM_F_SNAPSHOT | MPM_F_SIGW | MPM_F_EPSW | MPM_F_VW | MPM_F_N)
int mpm_snapshot(mpm_handle *h, mpm_h5 *f, int64_t group, double Ti, uint32_t field_mask, int32_t type);
int mpm_snapshot_wait(mpm_handle *h, int64_t *written);

/* ---- diagnostics ---- */
/* sizeof(mpm_desc), sizeof(mpm_view), sizeof(mpm_host_views), sizeof(mpm_stats):
 * lets a binding verify its struct layouts against the library's. */
int mpm_abi_sizes(int64_t *desc, int64_t *view, int64_t *views, int64_t *stats);
int mpm_get_stats(mpm_handle *h, mpm_stats *out);
const char *mpm_last_error(mpm_handle *h);
/* Triad bandwidth probe (Tpeak): bytes moved / best time, GB/s. */
int mpm_peak_bandwidth(int32_t device, double *gbs_out);
/* Profiling mode (mpm_set_profiling): every launch of a mpm_step call is
 * bracketed by events and waited for (no graph replay).  mpm_get_kernel_times
 * returns, per kernel name, the average device time per launch (ms) and the
 * launch count over the last mpm_step call, up to `cap` names. */
int mpm_set_profiling(mpm_handle *h, int32_t on);
int mpm_get_kernel_times(mpm_handle *h, const char **names, double *ms, int64_t *launches,
                         int32_t cap, int32_t *count);

#ifdef __cplusplus
}
#endif
#endif /* MPM_B200_H */
