// mpm_b200.cu -- C ABI (include/mpm_b200.h) of the B200 uGIMP MPM step.
//
// Host orchestration: device memory layout, upload/download of the
// reference's column-major host arrays, the per-step launch sequence and the
// cell sort.  Kernels live in mpm_kernels.cuh / mpm_sort.cuh.
#include "../../include/mpm_b200.h"
#include "mpm_tiled.cuh"
#include "mpm_box.cuh"
#include "mpm_ts.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

using namespace mpm;

namespace {

struct Err {
    int code;
    std::string msg;
};

#define CK(call)                                                                           \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            throw Err{MPM_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)};     \
    } while (0)

#define LAUNCH_CHECK()                                                                     \
    do {                                                                                   \
        cudaError_t e_ = cudaGetLastError();                                               \
        if (e_ != cudaSuccess) throw Err{MPM_E_CUDA, std::string("launch: ") + cudaGetErrorString(e_)}; \
    } while (0)

inline int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }

struct KTimer {
    const char *name;
    double ms = 0;
    int64_t n = 0;
};

// The tile shapes the autotuner tries (32 cells, one warp lane per cell; the
// box passes are compiled for these), default first.
struct TileShape {
    int tx, ty, tz;
};
inline std::vector<TileShape> tile_shapes(int dim) {
    if (dim == 3) return {{2, 8, 2}, {4, 8, 1}, {4, 4, 2}};
    return {{4, 8, 1}, {2, 16, 1}};
}

}  // namespace

namespace mpm_detail {
cudaError_t mlp_forward_prepare();
cudaError_t mlp_forward_dev(const float *P, const float *norm, const float *feat, float *out, int64_t cap,
                            const uint32_t *n_dev, int residual, int *err, cudaStream_t st, int nsm);
}

struct GraphCache {
    cudaGraphExec_t exec = nullptr;
    double dt = 0;
    void *pbuf0 = nullptr;
    int sort_every = 0;
    bool tiled = false, box = false, wide = false;
    int surr_mode = 0;
    int tile = 0;   // tx | ty << 8 | tz << 16
    int64_t launches = 0, steps = 0, sorts = 0;
};

// Snapshots in flight (mpm_snapshot): two slots, each a device buffer the
// un-permuting gather writes and a pinned host buffer the copy stream fills;
// a writer thread puts a slot into the file once its copy finished.
struct SnapJob {
    int slot;
    mpm_h5 *file;
    int64_t group;
    double Ti;
    uint32_t mask;
    int32_t type;
};
struct SnapState {
    cudaStream_t copy = nullptr;
    cudaEvent_t gathered[2] = {nullptr, nullptr}, copied[2] = {nullptr, nullptr};
    void *dev[2] = {nullptr, nullptr}, *host[2] = {nullptr, nullptr};
    size_t cap = 0;
    bool busy[2] = {false, false};
    int next = 0;
    int device = 0;
    int64_t np = 0;
    int dim = 3;
    std::thread th;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<SnapJob> q;
    bool stop = false;
    int err = MPM_OK;
    std::string msg;
    int64_t written = 0;
};

struct mpm_handle {
    mpm_desc d{};
    std::string last_error;
    cudaStream_t stream = nullptr;
    int dev = 0;
    bool fp64 = false;
    bool uploaded = false;
    bool coh_mode = false;   // per-particle cohesion (materials differ only in c)
    bool use_graphs = true;  // replay captured step blocks (MPM_B200_GRAPHS=0 turns it off)
    bool prefetch = true;    // FP32 particle pass stages fields by cp.async (MPM_B200_PREFETCH=0 turns it off)
    bool cell_major = false; // order inside a tile: rank-major (default) or cell-major (MPM_B200_ORDER=cell)
    bool chain = true;       // FP32 scatters merge chained warp lanes (MPM_B200_CHAIN=0 turns it off)
    bool box = false;        // FP32 MUSL passes with the tile's nodes in shared memory (variant 2; MPM_B200_BOX=1)
    bool wide = false;       // variant 3: the lane-merged fused pass at 3 resident CTAs per SM (85 registers; the 3D default)
    uint32_t *work = nullptr;   // tile counters of the box passes
    GraphCache graph;
    int64_t graph_launches = 0;
    // stress-return surrogate: 1 = log samples into caller buffers, 2 = infer
    int surr_mode = 0;
    mpm::SurrCtx surr{};
    float *surr_params = nullptr, *surr_norm = nullptr, *surr_out = nullptr, *surr_feat = nullptr;
    uint32_t *surr_cnt = nullptr, *surr_list = nullptr;
    float *surr_s0 = nullptr;   // deferred Mohr-Coulomb rows: rotated pre-increment stress (np x 6)
    unsigned long long *surr_stats = nullptr;   // rows deferred, fallbacks
    int *surr_err = nullptr;
    float surr_tol = 1e-3f, surr_sref = 1e3f;
    int surr_residual = 0;   // the network predicts the correction to the trial stress
    bool acc_valid = false;     // grid accumulators hold the P2G of the current particles
    double acc_Ti = 0.0;
    int64_t steps_done = 0, sorts_done = 0, since_sort = 1 << 30;
    int sort_every = 16;
    int err_host = 0;
    double last_step_ms = 0;
    size_t bytes = 0;
    std::vector<void *> allocs;
    // particle arrays: two copies (A = current, B = sort target)
    void *pbuf[2] = {nullptr, nullptr};
    // grid
    void *acc = nullptr, *gat = nullptr, *gvs = nullptr;   // node records (see mpm_kernels.cuh)
    bool ts = false;                                         // two-phase coupling (mpm_ts.cuh)
    void *accw = nullptr, *accd = nullptr, *gatw = nullptr, *bcvalw = nullptr;
    uint8_t *bcmask = nullptr;
    void *bcval = nullptr;
    void *csigm = nullptr, *comega = nullptr;   // MVL cell sums (R), nc each
    uint32_t *pcell = nullptr;                   // MVL start-of-step cell per particle
    int64_t nc = 0;
    uint32_t *bflag = nullptr;   // per node block: touched by a particle window
    uint32_t *blist = nullptr;   // list of the flagged blocks
    uint32_t *bcount = nullptr;  // its length
    int nbx = 1, nby = 1, nbz = 1;
    int64_t ni = 0;
    void *mat = nullptr;
    int *err = nullptr;
    // sort
    uint32_t *keys = nullptr, *cnt = nullptr, *off = nullptr, *bsum = nullptr, *big = nullptr, *nbig = nullptr;
    uint2 *pairs = nullptr, *pairs2 = nullptr;
    uint32_t nk = 0, big_cap = 0, nk_cap = 0;
    uint32_t *tiles = nullptr, *ntiles = nullptr;
    uint32_t ntile_total = 0;
    int nsm = 148;
    bool tiled = false;
    SortGeom sg{};
    size_t pbuf_size = 0;   // bytes of each particle buffer
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    bool profiling = false;
    std::vector<KTimer> ktimes;
    std::vector<cudaEvent_t> kev;
    int kernels_per_step = 4;
    int64_t launches = 0;
    SnapState *snap = nullptr;
};

namespace {

void *dalloc(mpm_handle *h, size_t bytes) {
    void *p = nullptr;
    CK(cudaMalloc(&p, bytes ? bytes : 16));
    h->allocs.push_back(p);
    h->bytes += bytes;
    return p;
}

template <int D, typename R> PDev<D, R> pdev_from(mpm_handle *h, int which) {
    PDev<D, R> P{};
    const int64_t np = h->d.np;
    char *b = (char *)h->pbuf[which];
    auto take = [&](size_t elem) {
        char *p = b;
        b += ((np * elem + 255) / 256) * 256;
        return (void *)p;
    };
    for (int d = 0; d < 3; ++d) P.x[d] = d < D ? (double *)take(8) : nullptr;
    for (int d = 0; d < 3; ++d) P.v[d] = d < D ? (R *)take(sizeof(R)) : nullptr;
    for (int c = 0; c < 6; ++c) P.sig[c] = c < PDev<D, R>::NV ? (R *)take(sizeof(R)) : nullptr;
    for (int c = 0; c < 9; ++c) P.F[c] = c < PDev<D, R>::NF ? (R *)take(sizeof(R)) : nullptr;
    for (int c = 0; c < 6; ++c) P.eps[c] = c < PDev<D, R>::NV ? (R *)take(sizeof(R)) : nullptr;
    P.epsq = (R *)take(sizeof(R));
    P.epsk = (R *)take(sizeof(R));
    P.epsv = (R *)take(sizeof(R));
    P.m = (R *)take(sizeof(R));
    P.vol0 = (R *)take(sizeof(R));
    P.vol = (R *)take(sizeof(R));
    P.mat = (uint32_t *)take(4);
    P.orig = (uint32_t *)take(4);
    R *coh = (R *)take(sizeof(R));
    P.coh = h->coh_mode ? coh : nullptr;
    if (h->ts) {
        P.n = (R *)take(sizeof(R));
        P.sigw = (R *)take(sizeof(R));
        P.mw = (R *)take(sizeof(R));
        for (int d = 0; d < 3; ++d) P.vw[d] = d < D ? (R *)take(sizeof(R)) : nullptr;
        for (int c = 0; c < 6; ++c) P.epsw[c] = c < PDev<D, R>::NV ? (R *)take(sizeof(R)) : nullptr;
    }
    return P;
}

size_t pbuf_bytes(int D, bool fp64, int64_t np, bool ts) {
    size_t R = fp64 ? 8 : 4;
    size_t per = 0;
    auto add = [&](size_t elem, int count) { per += count * (((np * elem + 255) / 256) * 256); };
    int NV = D == 2 ? 4 : 6;
    add(8, D);
    add(R, D);
    add(R, NV);
    add(R, D * D);
    add(R, NV);
    add(R, 7);
    add(4, 2);
    if (ts) {
        add(R, 3);      // n, σw, mw
        add(R, D);      // vw
        add(R, NV);     // ϵijw
    }
    return per;
}

template <typename R> GDev<R> gdev_from(mpm_handle *h) {
    using T4 = typename Vec<R>::T4;
    GDev<R> g{};
    const mpm_desc &d = h->d;
    double x1[3] = {d.x1, d.y1, d.z1}, hh[3] = {d.dx, d.dy, d.dz}, lp[3] = {d.lpx, d.lpy, d.lpz};
    int64_t nn[3] = {d.nnx, d.nny, d.dim == 3 ? d.nnz : 1};
    for (int a = 0; a < 3; ++a) {
        AxisC<R> &c = g.ax[a];
        c.x1 = x1[a];
        c.h = hh[a];
        c.inv_h = 1.0 / hh[a];
        c.supp = hh[a] + 0.5 * lp[a];
        c.hr = (R)hh[a];
        c.lp = (R)lp[a];
        c.half_lp = (R)(0.5 * lp[a]);
        c.h_m_hl = (R)(hh[a] - 0.5 * lp[a]);
        c.h_p_hl = (R)(hh[a] + 0.5 * lp[a]);
        c.invhl = (R)(1.0 / (hh[a] * lp[a]));
        c.invh = (R)(1.0 / hh[a]);
        c.nn = (int)nn[a];
        c.nc = (int)std::max<int64_t>(nn[a] - 1, 1);
    }
    g.nnx = (int)nn[0];
    g.nny = (int)nn[1];
    g.nnz = (int)nn[2];
    g.acc = (Node8<R> *)h->acc;
    g.gat = (Node8<R> *)h->gat;
    g.gvs = (T4 *)h->gvs;
    g.bcmask = h->bcmask;
    g.bcval = (const T4 *)h->bcval;
    g.mat = (const Mat<R> *)h->mat;
    g.err = h->err;
    g.csigm = (R *)h->csigm;
    g.comega = (R *)h->comega;
    g.pcell = h->pcell;
    g.bflag = h->bflag;
    g.blist = h->blist;
    g.bcount = h->bcount;
    g.nbx = h->nbx;
    g.nby = h->nby;
    g.nbz = h->nbz;
    g.accw = (Node8<R> *)h->accw;
    g.accd = (T4 *)h->accd;
    g.gatw = (Node8<R> *)h->gatw;
    g.bcvalw = (const T4 *)h->bcvalw;
    return g;
}

// ---- host type conversion helpers -------------------------------------------------
double view_get(const mpm_view &v, int64_t i, int64_t k) {
    int64_t idx = i + v.ld * k;
    switch (v.type) {
        case MPM_T_F64: return ((const double *)v.ptr)[idx];
        case MPM_T_F32: return ((const float *)v.ptr)[idx];
        case MPM_T_I64: return (double)((const int64_t *)v.ptr)[idx];
        case MPM_T_I32: return (double)((const int32_t *)v.ptr)[idx];
    }
    return 0.0;
}
int64_t view_geti(const mpm_view &v, int64_t i) {
    switch (v.type) {
        case MPM_T_I64: return ((const int64_t *)v.ptr)[i];
        case MPM_T_I32: return ((const int32_t *)v.ptr)[i];
        case MPM_T_F64: return (int64_t)((const double *)v.ptr)[i];
        case MPM_T_F32: return (int64_t)((const float *)v.ptr)[i];
    }
    return 0;
}
size_t type_size(int t) { return (t == MPM_T_F64 || t == MPM_T_I64) ? 8 : 4; }

// device-side conversion of one staged host column into a state array
template <typename S, typename T>
__global__ void k_convert(const S *src, T *dst, int64_t n) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = (T)src[i];
}
// scatter a state array into original order with conversion
template <typename S, typename T>
__global__ void k_unpermute(const S *src, const uint32_t *orig, T *dst, int64_t n) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[orig[i]] = (T)src[i];
}
__global__ void k_iota(uint32_t *a, int64_t n) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = (uint32_t)i;
}
template <int D, typename R>
__global__ void k_derived(PDev<D, R> P, int64_t np, int what, double *out) {
    // what: 0 Ω = det(F) Ω0 (FP64 det), 1 σm, 2 ρs = ρs0 / J, with ρs0 = m / Ω0,
    // 3 ρw = mw / Ω (two-phase)
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    double v = 0;
    if (what == 3) {
        v = (double)P.mw[i] / (double)P.vol[i];
    } else if (what == 1) {
        v = (double)((P.sig[0][i] + P.sig[1][i] + P.sig[2][i]) * (R)0.333333);
    } else {
        double J;
        if (D == 2) {
            J = (double)P.F[0][i] * (double)P.F[3][i] - (double)P.F[1][i] * (double)P.F[2][i];
        } else {
            double g[9];
            for (int k = 0; k < 9; ++k) g[k] = (double)P.F[k][i];
            J = g[0] * g[4] * g[8] + g[1] * g[5] * g[6] + g[2] * g[3] * g[7] - g[6] * g[4] * g[2] -
                g[7] * g[5] * g[0] - g[8] * g[3] * g[1];
        }
        if (what == 0) v = (double)P.vol[i];
        else v = ((double)P.m[i] / (double)P.vol0[i]) / J;
    }
    out[P.orig[i]] = v;
}

// Synchronises a stream when it leaves scope (host buffers of pending copies).
struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() { cudaStreamSynchronize(s); }
};

// Host <-> device staging.  The sort's target buffer (pbuf[1]) holds nothing
// between sorts, and every staged copy below is ordered on h->stream with the
// sorts, so it serves as the staging area: at least 24 bytes per particle
// (positions alone take 8 per axis), i.e. three FP64 columns.
char *stage_area(mpm_handle *h, size_t bytes) {
    if (bytes > h->pbuf_size) throw Err{MPM_E_ARG, "staging request larger than a particle buffer"};
    return (char *)h->pbuf[1];
}

// Stage host column k of view v (any element type) into the first np x 8
// bytes of the staging area and convert it into dst.  No host synchronisation:
// the staging slot is reused only by later work on the same stream, and the
// caller synchronises once after its last copy.
template <typename T>
void upload_col(mpm_handle *h, const mpm_view &v, int64_t k, T *dst, int64_t n) {
    size_t es = type_size(v.type);
    char *stage = stage_area(h, n * 8);
    const char *src = (const char *)v.ptr + (size_t)(v.ld * k) * es;
    CK(cudaMemcpyAsync(stage, src, n * es, cudaMemcpyHostToDevice, h->stream));
    int64_t nb = cdiv(n, 256);
    switch (v.type) {
        case MPM_T_F64: k_convert<double, T><<<nb, 256, 0, h->stream>>>((const double *)stage, dst, n); break;
        case MPM_T_F32: k_convert<float, T><<<nb, 256, 0, h->stream>>>((const float *)stage, dst, n); break;
        case MPM_T_I64: k_convert<long long, T><<<nb, 256, 0, h->stream>>>((const long long *)stage, dst, n); break;
        case MPM_T_I32: k_convert<int, T><<<nb, 256, 0, h->stream>>>((const int *)stage, dst, n); break;
    }
    LAUNCH_CHECK();
}

// Download a state array in original order into host column k of view v.
// A copy into pageable host memory returns once it has landed; into pinned
// memory it is asynchronous and the caller synchronises after its last copy.
template <typename S>
void download_col(mpm_handle *h, const S *src, const uint32_t *orig, const mpm_view &v, int64_t k, int64_t n) {
    size_t es = type_size(v.type);
    char *stage = stage_area(h, n * 8);
    int64_t nb = cdiv(n, 256);
    if (v.type == MPM_T_F64) k_unpermute<S, double><<<nb, 256, 0, h->stream>>>(src, orig, (double *)stage, n);
    else if (v.type == MPM_T_F32) k_unpermute<S, float><<<nb, 256, 0, h->stream>>>(src, orig, (float *)stage, n);
    else throw Err{MPM_E_ARG, "float field requested into an integer view"};
    LAUNCH_CHECK();
    char *dst = (char *)v.ptr + (size_t)(v.ld * k) * es;
    CK(cudaMemcpyAsync(dst, stage, n * es, cudaMemcpyDeviceToHost, h->stream));
}

// m = (R)(a * b) from two staged FP64 columns: the particle mass Ω·ρ rounded
// once from FP64, as the host product would be
template <typename R>
__global__ void k_mass(const double *a, const double *b, R *m, int64_t n) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) m[i] = (R)(a[i] * b[i]);
}

// ---- materials ---------------------------------------------------------------------
// M is the caller's: it must outlive the asynchronous copy
template <typename R> void build_materials(mpm_handle *h, const mpm_host_views *v, std::vector<Mat<R>> &M) {
    const int64_t nm = h->coh_mode ? 1 : h->d.nmat;
    M.assign(nm, Mat<R>{});
    auto get = [&](const mpm_view &vw, int64_t i) { return vw.ptr ? view_get(vw, i, 0) : 0.0; };
    for (int64_t i = 0; i < nm; ++i) {
        double K = get(v->Ks, i), G = get(v->Gs, i), c = get(v->c, i), phi = get(v->phi, i),
               psi = get(v->psi, i), sigt = get(v->sigt, i), Hp = get(v->Hp, i), cr = get(v->cr, i);
        Mat<R> &m = M[i];
        std::memset(&m, 0, sizeof(m));
        m.K = (R)K; m.G = (R)G;
        // constants as written in linearelastic.jl:48-49
        m.Dt = (R)(K + 1.333333 * G);
        m.Dd = (R)(K - 0.666667 * G);
        m.c = (R)c; m.phi = (R)phi; m.psi = (R)psi; m.sigt = (R)sigt; m.Hp = (R)Hp; m.cr = (R)cr;
        // druckerprager.jl:39-44, 59
        double kphi = (6.0 * c * std::cos(phi)) / (1.732051 * (3.0 + std::sin(phi)));
        double qphi = (6.0 * std::sin(phi)) / (1.732051 * (3.0 + std::sin(phi)));
        double qpsi = (6.0 * std::sin(psi)) / (1.732051 * (3.0 + std::sin(psi)));
        double st = std::min(sigt, kphi / qphi);
        m.kphi = (R)kphi; m.qphi = (R)qphi; m.qpsi = (R)qpsi; m.st = (R)st;
        m.ab = (R)(std::sqrt(1.0 + qphi * qphi) - qphi);
        m.tb = (R)(kphi - qphi * st);
        m.dq = (R)std::sqrt(0.333333 + 0.222222 * qpsi * qpsi);
        m.sphi = (R)std::sin(phi); m.cphi = (R)std::cos(phi); m.tphi = (R)std::tan(phi);
        m.spsi = (R)std::sin(psi); m.tpsi = (R)std::tan(psi);
        m.kc = (R)((6.0 * std::cos(phi)) / (1.732051 * (3.0 + std::sin(phi))));
        if (h->ts) {
            m.Kw = (R)get(v->Kw, v->Kw.ld > i ? i : 0);
            m.kperm = (R)get(v->kperm, v->kperm.ld > i ? i : 0);
            if (!(m.kperm != R(0))) throw Err{MPM_E_ARG, "two-phase model needs a non-zero permeability k"};
        }
    }
    CK(cudaMemcpyAsync(h->mat, M.data(), nm * sizeof(Mat<R>), cudaMemcpyHostToDevice, h->stream));
}

// ---- profiling mode: device time of a span of the library stream, by name ---------
void prof_begin(mpm_handle *h) {
    if (h->kev.size() < 2) {
        cudaEvent_t a, b;
        CK(cudaEventCreate(&a));
        CK(cudaEventCreate(&b));
        h->kev.push_back(a);
        h->kev.push_back(b);
    }
    CK(cudaEventRecord(h->kev[0], h->stream));
}
void prof_end(mpm_handle *h, const char *name) {
    KTimer *kt = nullptr;
    for (KTimer &k : h->ktimes)
        if (std::strcmp(k.name, name) == 0) { kt = &k; break; }
    if (!kt) {
        h->ktimes.push_back(KTimer{name});
        kt = &h->ktimes.back();
    }
    CK(cudaEventRecord(h->kev[1], h->stream));
    CK(cudaEventSynchronize(h->kev[1]));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, h->kev[0], h->kev[1]));
    kt->ms += ms;
    kt->n += 1;
}

// ---- the sort ----------------------------------------------------------------------
template <int D, typename R> void do_sort(mpm_handle *h) {
    const int64_t np = h->d.np;
    if (np == 0) return;
    if (h->profiling) prof_begin(h);
    cudaStream_t st = h->stream;
    PDev<D, R> A = pdev_from<D, R>(h, 0), B = pdev_from<D, R>(h, 1);
    GDev<R> g = gdev_from<R>(h);
    CK(cudaMemsetAsync(h->cnt, 0, (size_t)h->nk * 4, st));
    k_sort_keys<D, R><<<cdiv(np, 256), 256, 0, st>>>(A, g, h->sg, np, h->keys, h->cnt);
    LAUNCH_CHECK();
    uint32_t nb = (uint32_t)cdiv(h->nk, SCAN_CHUNK);
    k_scan_reduce<<<nb, SCAN_T, 0, st>>>(h->cnt, h->nk, h->bsum);
    k_scan_top<<<1, SCAN_T, 0, st>>>(h->bsum, nb);
    k_scan_down<<<nb, SCAN_T, 0, st>>>(h->cnt, h->nk, h->bsum, h->off);
    LAUNCH_CHECK();
    CK(cudaMemsetAsync(h->cnt, 0, (size_t)h->nk * 4, st));
    CK(cudaMemsetAsync(h->nbig, 0, 4, st));
    k_sort_scatter<D, R><<<cdiv(np, 256), 256, 0, st>>>(A, np, h->keys, h->off, h->cnt, h->pairs);
    k_sort_buckets<<<cdiv(h->nk, 256), 256, 0, st>>>(h->off, h->nk, h->pairs, h->big, h->nbig, h->big_cap, h->err);
    k_sort_big<<<64, 512, 0, st>>>(h->off, h->big, h->nbig, h->big_cap, h->pairs);
    CK(cudaMemsetAsync(h->ntiles, 0, 4, st));
    const int cpt = h->sg.cpt;
    k_tile_list<<<cdiv(h->ntile_total, 256), 256, 0, st>>>(h->off, h->ntile_total, (uint32_t)cpt, h->tiles, h->ntiles);
    if (h->cell_major) {
        // particles of a cell stay consecutive (tile-major, then cell, then (octant, original index))
        k_permute<D, R><<<cdiv(np, 256), 256, 0, st>>>(A, B, h->pairs, np);
    } else {
        if (cpt == 32)
            k_tile_transpose<32><<<h->nsm * 16, 32, 0, st>>>(h->off, h->tiles, h->ntiles, h->pairs, h->pairs2);
        else if (cpt == 64)
            k_tile_transpose<64><<<h->nsm * 16, 64, 0, st>>>(h->off, h->tiles, h->ntiles, h->pairs, h->pairs2);
        else
            k_tile_transpose<128><<<h->nsm * 8, 128, 0, st>>>(h->off, h->tiles, h->ntiles, h->pairs, h->pairs2);
        k_permute<D, R><<<cdiv(np, 256), 256, 0, st>>>(A, B, h->pairs2, np);
    }
    LAUNCH_CHECK();
    std::swap(h->pbuf[0], h->pbuf[1]);
    h->since_sort = 0;
    h->sorts_done++;
    h->launches += 10;
    if (h->profiling) prof_end(h, "sort");
}

// ---- step --------------------------------------------------------------------------
// Issues one pass.  In profiling mode each launch is bracketed by events on the
// library stream and waited for, and its time is added to the per-kernel
// totals under its name (the launch sequence of a call varies: the standalone
// P2G, the sorts).
struct Launcher {
    mpm_handle *h;
    template <typename F> void run(const char *name, F &&f) {
        if (h->profiling) {
            prof_begin(h);
            f();
            LAUNCH_CHECK();
            prof_end(h, name);
        } else {
            f();
            LAUNCH_CHECK();
        }
        ++h->launches;
    }
};

double gravity_at(const mpm_desc &d, double Ti) {
    // OS_MUSL.jl:70: G = Ti < Te ? gravity / Te * Ti : gravity
    return Ti < d.Te ? d.gravity / d.Te * Ti : d.gravity;
}

// dynamic shared memory of the particle pass (staged particle fields)
inline size_t g2p_smem(const StepParams &sp) { return sp.prefetch ? (size_t)PF_N * PF_T * sizeof(float) : 0; }

template <int D, typename R> StepParams make_params(mpm_handle *h, double dt, double Ti, double Gscatter) {
    StepParams sp{};
    sp.dt = dt;
    sp.G = Gscatter;
    sp.FLIP = h->d.FLIP;
    sp.PIC = h->d.PIC;
    sp.zeta = h->d.zeta_s;
    sp.plastic = Ti >= h->d.Te;
    sp.constitutive = h->d.constitutive;
    sp.mc3d = h->d.mc3d == MPM_MC3D_RESTATED ? 1 : 0;
    sp.va = h->d.va;
    sp.usl = h->d.scheme == MPM_SCHEME_USL ? 1 : 0;
    sp.prefetch = (sizeof(R) == 4 && h->prefetch) ? 1 : 0;
    // grid vs is gathered by the :v updates and by the PIC term of MUSL :a (USL :a
    // maps the updated velocity, which is the vsT record)
    sp.need_vs = (h->d.va == MPM_VA_V || (h->d.PIC != 0.0 && !sp.usl)) ? 1 : 0;
    sp.np = h->d.np;
    sp.mvl = h->d.mvl ? 1 : 0;
    sp.ts = h->ts ? 1 : 0;
    sp.zeta_w = h->d.zeta_w;
    // massless-node cutoff m < eps(T2) of the solves (utils_OS.jl:515, 555, 975): T2
    // is the reference's float type (the user's ϵ), whatever the device stores
    sp.meps = h->d.time_f32 ? 1.1920928955078125e-07 : 2.220446049250313e-16;
    sp.surr = h->surr;
    sp.surr.mode = (D == 3 && !h->ts && (h->d.constitutive == MPM_DRUCKERPRAGER ||
                                          (h->d.constitutive == MPM_MOHRCOULOMB && h->d.mc3d == MPM_MC3D_RESTATED)))
                       ? h->surr_mode
                       : 0;
    sp.surr.salt = (uint32_t)(h->steps_done * 0x9E3779B9ull);
    return sp;
}

template <int D, typename R> void standalone_p2g(mpm_handle *h, double Ti, Launcher &L) {
    const int64_t np = h->d.np;
    using T4 = typename Vec<R>::T4;
    CK(cudaMemsetAsync(h->acc, 0, h->ni * sizeof(Node8<R>), h->stream));
    CK(cudaMemsetAsync(h->bflag, 0, (size_t)h->nbx * h->nby * h->nbz * 4, h->stream));
    CK(cudaMemsetAsync(h->bcount, 0, 4, h->stream));
    PDev<D, R> P = pdev_from<D, R>(h, 0);
    GDev<R> g = gdev_from<R>(h);
    StepParams sp = make_params<D, R>(h, 0.0, Ti, gravity_at(h->d, Ti));
    if (h->ts) {
        CK(cudaMemsetAsync(h->accw, 0, h->ni * sizeof(Node8<R>), h->stream));
        CK(cudaMemsetAsync(h->accd, 0, h->ni * sizeof(T4), h->stream));
        if (np) L.run("p2g", [&] { k_p2g_ts<D, R><<<cdiv(np, 256), 256, 0, h->stream>>>(P, g, sp); });
    } else if (np) {
        L.run("p2g", [&] { k_p2g<D, R><<<cdiv(np, 256), 256, 0, h->stream>>>(P, g, sp); });
    }
    h->acc_valid = true;
    h->acc_Ti = Ti;
}

struct TiledCfg {
    size_t smem_dm = 0, smem_g2p = 0;
    int grid_dm = 0, grid_g2p = 0;
    bool ready = false;
};

// dynamic shared memory and persistent grid size (CTAs per SM x SMs) of the tiled kernels
template <int D, typename R> const TiledCfg &tiled_cfg(mpm_handle *h, int need_vs) {
    static thread_local TiledCfg per[8][2];   // per device ordinal (mod 8) and need_vs
    TiledCfg &cc = per[h->dev & 7][need_vs ? 1 : 0];
    if (cc.ready) return cc;
    using W = Win<D>;
    cc.smem_dm = (size_t)(need_vs ? 9 : 6) * W::WN * sizeof(R);
    cc.smem_g2p = (size_t)6 * W::WN * sizeof(R);
    CK(cudaFuncSetAttribute(k_dmap_tile<D, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cc.smem_dm));
    CK(cudaFuncSetAttribute(k_g2p_tile<D, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cc.smem_g2p));
    CK(cudaFuncSetAttribute(k_g2p_tile<D, R, D == 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cc.smem_g2p));
    int a = 0, b = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_dmap_tile<D, R>, 256, cc.smem_dm));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_g2p_tile<D, R>, 256, cc.smem_g2p));
    cc.grid_dm = std::max(a, 1) * h->nsm;
    cc.grid_g2p = std::max(b, 1) * h->nsm;
    cc.ready = true;
    return cc;
}

// ---- box passes (mpm_box.cuh) ---------------------------------------------------------
// Tile shapes with compiled box passes (32 cells each).
#define MPM_BOX_SHAPES_3D(X) X(3, 2, 8, 2) X(3, 4, 8, 1) X(3, 4, 4, 2)
#define MPM_BOX_SHAPES_2D(X) X(2, 4, 8, 1) X(2, 2, 16, 1)

template <int D, int TX, int TY, int TZ> struct BoxPass {
    using G = BoxGeo<D, TX, TY, TZ>;
    static constexpr size_t G2P_SMEM = (size_t)MPM_BOX_WARPS * G::G2P_BYTES;
    static constexpr size_t DM_SMEM = (size_t)MPM_BOX_WARPS * G::DM_BYTES;
    static void prepare() {
        CK(cudaFuncSetAttribute(k_g2p_box<D, TX, TY, TZ, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)G2P_SMEM));
        if (D == 3)
            CK(cudaFuncSetAttribute(k_g2p_box<D, TX, TY, TZ, D == 3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)G2P_SMEM));
        CK(cudaFuncSetAttribute(k_dmap_box<D, TX, TY, TZ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)DM_SMEM));
    }
    static void dmap(mpm_handle *h, const PDev<D, float> &P, const GDev<float> &g, const StepParams &sp,
                     const BoxTiles &bt) {
        k_dmap_box<D, TX, TY, TZ><<<h->nsm * MPM_BOX_DMAP_MINB, MPM_BOX_WARPS * 32, DM_SMEM, h->stream>>>(P, g, sp,
                                                                                                        bt);
    }
    static void g2p(mpm_handle *h, const PDev<D, float> &P, const GDev<float> &g, const StepParams &sp,
                    const BoxTiles &bt, bool mc3) {
        if (mc3 && D == 3)
            k_g2p_box<D, TX, TY, TZ, D == 3><<<h->nsm * MPM_BOX_G2P_MINB, MPM_BOX_WARPS * 32, G2P_SMEM, h->stream>>>(
                P, g, sp, bt);
        else
            k_g2p_box<D, TX, TY, TZ, false><<<h->nsm * MPM_BOX_G2P_MINB, MPM_BOX_WARPS * 32, G2P_SMEM, h->stream>>>(
                P, g, sp, bt);
    }
};

int tile_code(const SortGeom &sg) { return sg.tx | sg.ty << 8 | sg.tz << 16; }

// Shared-memory limits of the box passes (outside any stream capture).
void box_prepare(mpm_handle *h) {
#define MPM_BOX_PREP(D, A, B, C) \
    if (h->d.dim == D) BoxPass<D, A, B, C>::prepare();
    MPM_BOX_SHAPES_3D(MPM_BOX_PREP)
    MPM_BOX_SHAPES_2D(MPM_BOX_PREP)
#undef MPM_BOX_PREP
}

// Does the handle's tile shape have box passes?
bool box_shape_ok(const mpm_handle *h) {
    const SortGeom &sg = h->sg;
#define MPM_BOX_HAS(D, A, B, C) \
    if (h->d.dim == D && sg.tx == A && sg.ty == B && (D == 2 || sg.tz == C)) return true;
    MPM_BOX_SHAPES_3D(MPM_BOX_HAS)
    MPM_BOX_SHAPES_2D(MPM_BOX_HAS)
#undef MPM_BOX_HAS
    return false;
}

// One box pass (which = 0: double mapping, 1: fused G2P + next P2G) with the
// handle's tile shape.
template <int D> void box_launch(mpm_handle *h, int which, const PDev<D, float> &P, const GDev<float> &g,
                                 const StepParams &sp, bool mc3) {
    BoxTiles bt{h->tiles, h->ntiles, h->off, h->work + which, h->sg};
    CK(cudaMemsetAsync(h->work + which, 0, 4, h->stream));
    const SortGeom &sg = h->sg;
#define MPM_BOX_GO(DD, A, B, C)                                                                 \
    if constexpr (D == DD) {                                                                    \
        if (sg.tx == A && sg.ty == B && (DD == 2 || sg.tz == C)) {                              \
            if (which == 0) BoxPass<DD, A, B, C>::dmap(h, P, g, sp, bt);                        \
            else BoxPass<DD, A, B, C>::g2p(h, P, g, sp, bt, mc3);                               \
            return;                                                                             \
        }                                                                                       \
    }
    MPM_BOX_SHAPES_3D(MPM_BOX_GO)
    MPM_BOX_SHAPES_2D(MPM_BOX_GO)
#undef MPM_BOX_GO
    throw Err{MPM_E_STATE, "no box pass for this tile shape"};
}

// The launches of one step (solve, double mapping, DM3, fused G2P + next P2G).
// the lane-merged double mapping, specialised for va = :a without the separate
// grid velocity (its gathers then read one half-record per node, no switches)
template <int D, typename R>
void launch_dmap_chain(mpm_handle *h, const PDev<D, R> &P, const GDev<R> &g, const StepParams &sp) {
    const int64_t np = sp.np;
    if (sp.va == MPM_VA_A && !sp.need_vs) k_dmap_chain<D, R, false><<<cdiv(np, 256), 256, 0, h->stream>>>(P, g, sp);
    else k_dmap_chain<D, R, true><<<cdiv(np, 256), 256, 0, h->stream>>>(P, g, sp);
}

template <int D, typename R> void issue_step(mpm_handle *h, Launcher &L, double dt, double Ti, double Tn) {
    const int64_t np = h->d.np;
    const int nblk = h->nbx * h->nby * h->nbz;
    const int ngrid = std::min(nblk, h->nsm * 16);   // node passes: grid-stride over the active-block list
    if (h->since_sort >= h->sort_every) do_sort<D, R>(h);
    PDev<D, R> P = pdev_from<D, R>(h, 0);
    GDev<R> g = gdev_from<R>(h);
    StepParams sp = make_params<D, R>(h, dt, Ti, gravity_at(h->d, Tn));
    const bool mc3 = sp.mc3d && sp.constitutive == MPM_MOHRCOULOMB;
    if (sp.ts) {
        // two-phase MUSL (TS_MUSL.jl): solve, DM1+DM2, DM3, G2P_TS! + next P2G_TS!
        L.run("solve", [&] { k_solve_ts<D, R><<<ngrid, Blk<D>::NT, 0, h->stream>>>(g, sp); });
        if (np) L.run("dmap", [&] {
            if (h->chain) k_dmap_ts_chain<D, R><<<cdiv(np, 256), 256, 0, h->stream>>>(P, g, sp);
            else k_dmap_ts<D, R><<<cdiv(np, 256), 256, 0, h->stream>>>(P, g, sp);
        });
        L.run("dm3", [&] { k_dm3_ts<D, R><<<ngrid, Blk<D>::NT, 0, h->stream>>>(g, sp); });
        CK(cudaMemsetAsync(h->bcount, 0, 4, h->stream));
        if (np) L.run("g2p_p2g", [&] {
            if (h->chain) {
                if (mc3) k_g2p_ts_chain<D, D == 3, R><<<cdiv(np, 256), 256, g2p_smem(sp), h->stream>>>(P, g, sp);
                else k_g2p_ts_chain<D, false, R><<<cdiv(np, 256), 256, g2p_smem(sp), h->stream>>>(P, g, sp);
                return;
            }
            if (mc3) k_g2p_ts<D, R, true, D == 3><<<cdiv(np, 256), 256, 0, h->stream>>>(P, g, sp);
            else k_g2p_ts<D, R, true><<<cdiv(np, 256), 256, 0, h->stream>>>(P, g, sp);
        });
        h->since_sort++;
        h->steps_done++;
        return;
    }
    L.run("solve", [&] { k_solve<D, R><<<ngrid, Blk<D>::NT, 0, h->stream>>>(g, sp); });
    if (h->tiled && !sp.mvl && !sp.usl && sp.surr.mode != 2) {
        TileList tl{h->tiles, h->ntiles, h->off, h->sg};
        const TiledCfg &c = tiled_cfg<D, R>(h, sp.need_vs);
        if (np) L.run("dmap", [&] { k_dmap_tile<D, R><<<c.grid_dm, 256, c.smem_dm, h->stream>>>(P, g, sp, tl); });
        L.run("dm3", [&] { k_dm3<D, R><<<ngrid, Blk<D>::NT, 0, h->stream>>>(g, sp); });
        CK(cudaMemsetAsync(h->bcount, 0, 4, h->stream));
        if (np) L.run("g2p_p2g", [&] {
            if (mc3) k_g2p_tile<D, R, D == 3><<<c.grid_g2p, 256, c.smem_g2p, h->stream>>>(P, g, sp, tl);
            else k_g2p_tile<D, R><<<c.grid_g2p, 256, c.smem_g2p, h->stream>>>(P, g, sp, tl);
        });
    } else if (sp.usl && np) {
        // USL: no double mapping; DM1 (velocity, position) rides in the G2P pass
        CK(cudaMemsetAsync(h->bcount, 0, 4, h->stream));
        if (sp.mvl) {
            CK(cudaMemsetAsync(h->csigm, 0, (size_t)h->nc * sizeof(R), h->stream));
            CK(cudaMemsetAsync(h->comega, 0, (size_t)h->nc * sizeof(R), h->stream));
            L.run("g2p", [&] {
                if (mc3) k_g2p<D, R, false, D == 3, true><<<cdiv(np, 256), 256, g2p_smem(sp), h->stream>>>(P, g, sp);
                else k_g2p<D, R, false, false, true><<<cdiv(np, 256), 256, g2p_smem(sp), h->stream>>>(P, g, sp);
            });
            L.run("mvl_p2g", [&] {
                if (h->chain) k_mvl_p2g_chain<D, R><<<cdiv(np, 256), 256, 0, h->stream>>>(P, g, sp);
                else k_mvl_p2g<D, R><<<cdiv(np, 256), 256, 0, h->stream>>>(P, g, sp);
            });
        } else {
            L.run("g2p_p2g", [&] {
                if (h->chain) {
                    if (mc3) k_g2p_chain<D, D == 3, true, R><<<cdiv(np, 256), 256, g2p_smem(sp), h->stream>>>(P, g, sp);
                    else k_g2p_chain<D, false, true, R><<<cdiv(np, 256), 256, g2p_smem(sp), h->stream>>>(P, g, sp);
                    return;
                }
                if (mc3) k_g2p<D, R, true, D == 3, true><<<cdiv(np, 256), 256, g2p_smem(sp), h->stream>>>(P, g, sp);
                else k_g2p<D, R, true, false, true><<<cdiv(np, 256), 256, g2p_smem(sp), h->stream>>>(P, g, sp);
            });
        }
    } else if (sp.mvl && np) {
        // MVL: update + cell sums, then the cell-averaged mean stress + P2G
        // (the scatters of chained lanes merged, as in the default passes)
        const bool chain = h->chain;
        L.run("dmap", [&] {
            if (chain) launch_dmap_chain<D, R>(h, P, g, sp);
            else k_dmap<D, R><<<cdiv(np, 256), 256, 0, h->stream>>>(P, g, sp);
        });
        L.run("dm3", [&] { k_dm3<D, R><<<ngrid, Blk<D>::NT, 0, h->stream>>>(g, sp); });
        CK(cudaMemsetAsync(h->bcount, 0, 4, h->stream));
        CK(cudaMemsetAsync(h->csigm, 0, (size_t)h->nc * sizeof(R), h->stream));
        CK(cudaMemsetAsync(h->comega, 0, (size_t)h->nc * sizeof(R), h->stream));
        L.run("g2p", [&] {
            if (mc3) k_g2p<D, R, false, D == 3><<<cdiv(np, 256), 256, g2p_smem(sp), h->stream>>>(P, g, sp);
            else k_g2p<D, R, false><<<cdiv(np, 256), 256, g2p_smem(sp), h->stream>>>(P, g, sp);
        });
        L.run("mvl_p2g", [&] {
            if (chain) k_mvl_p2g_chain<D, R><<<cdiv(np, 256), 256, 0, h->stream>>>(P, g, sp);
            else k_mvl_p2g<D, R><<<cdiv(np, 256), 256, 0, h->stream>>>(P, g, sp);
        });
    } else if (sp.surr.mode == 2 && sp.plastic && np) {
        // surrogate: G2P + update with the yielding particles' returns deferred,
        // the MLP over the deferred rows, accept-or-fallback, then the scatter
        L.run("dmap", [&] { launch_dmap_chain<D, R>(h, P, g, sp); });
        L.run("dm3", [&] { k_dm3<D, R><<<ngrid, Blk<D>::NT, 0, h->stream>>>(g, sp); });
        CK(cudaMemsetAsync(h->bcount, 0, 4, h->stream));
        CK(cudaMemsetAsync(h->surr_cnt, 0, 4, h->stream));
        // the fused pass: particles whose return is deferred skip its scatter
        L.run("g2p_p2g", [&] {
            if (mc3) k_g2p_chain<D, D == 3, false, R><<<cdiv(np, 256), 256, g2p_smem(sp), h->stream>>>(P, g, sp);
            else k_g2p_chain<D, false, false, R><<<cdiv(np, 256), 256, g2p_smem(sp), h->stream>>>(P, g, sp);
        });
        L.run("mlp", [&] {
            CK(mpm_detail::mlp_forward_dev(h->surr_params, h->surr_norm, h->surr_feat, h->surr_out, np, h->surr_cnt,
                                           h->surr_residual, h->surr_err, h->stream, h->nsm));
        });
        if constexpr (D == 3) {
            L.run("surr_fix", [&] {
                if (mc3)
                    k_surr_fix_mc<R><<<h->nsm * 8, 256, 0, h->stream>>>(P, g, sp.surr, h->surr_out, h->surr_tol,
                                                                     h->surr_sref, h->surr_stats);
                else
                    k_surr_fix<R><<<h->nsm * 8, 256, 0, h->stream>>>(P, g, sp.surr, h->surr_out, h->surr_tol,
                                                                  h->surr_sref, h->surr_stats);
            });
        }
        L.run("p2g", [&] {
            k_p2g_list<D, R><<<h->nsm * 8, 256, 0, h->stream>>>(P, g, sp, h->surr_list, h->surr_cnt, (uint32_t)np);
        });
    } else if (std::is_same<R, float>::value && h->box && sp.va == MPM_VA_A && !sp.need_vs && box_shape_ok(h)) {
        // FP32 MUSL :a: the box passes (node data of a tile in shared memory)
        if constexpr (std::is_same<R, float>::value) {
            if (np) L.run("dmap", [&] { box_launch<D>(h, 0, P, g, sp, mc3); });
            L.run("dm3", [&] { k_dm3<D, R><<<ngrid, Blk<D>::NT, 0, h->stream>>>(g, sp); });
            CK(cudaMemsetAsync(h->bcount, 0, 4, h->stream));
            if (np) L.run("g2p_p2g", [&] { box_launch<D>(h, 1, P, g, sp, mc3); });
        }
    } else {
        const bool chain = h->chain;
        if (np) L.run("dmap", [&] {
            if (chain) launch_dmap_chain<D, R>(h, P, g, sp);
            else k_dmap<D, R><<<cdiv(np, 256), 256, 0, h->stream>>>(P, g, sp);
        });
        L.run("dm3", [&] { k_dm3<D, R><<<ngrid, Blk<D>::NT, 0, h->stream>>>(g, sp); });
        CK(cudaMemsetAsync(h->bcount, 0, 4, h->stream));
        if (np) L.run("g2p_p2g", [&] {
            if (chain) {
                if (mc3) k_g2p_chain<D, D == 3, false, R><<<cdiv(np, 256), 256, g2p_smem(sp), h->stream>>>(P, g, sp);
                else if (h->wide) k_g2p_chain<D, false, false, R, 3><<<cdiv(np, 256), 256, g2p_smem(sp), h->stream>>>(P, g, sp);
                else k_g2p_chain<D, false, false, R><<<cdiv(np, 256), 256, g2p_smem(sp), h->stream>>>(P, g, sp);
                return;
            }
            if (mc3) k_g2p<D, R, true, D == 3><<<cdiv(np, 256), 256, g2p_smem(sp), h->stream>>>(P, g, sp);
            else k_g2p<D, R, true><<<cdiv(np, 256), 256, g2p_smem(sp), h->stream>>>(P, g, sp);
        });
    }
    h->since_sort++;
    h->steps_done++;
}

// Steps after the gravity ramp (Ti >= Te) all launch with the same parameters,
// so a block of two sort periods -- sort, S steps, sort, S steps, after which
// the ping-pong particle buffers are back in place -- is captured once into a
// CUDA graph and replayed.  The capture is keyed on everything baked into the
// launches; the host bookkeeping of a replay repeats what the capture did.
template <int D, typename R> bool graph_block(mpm_handle *h, double dt, double Ti) {
    GraphCache &gc = h->graph;
    const int S = h->sort_every;
    const bool match = gc.exec && gc.dt == dt && gc.pbuf0 == h->pbuf[0] && gc.sort_every == S &&
                       gc.tiled == h->tiled && gc.box == h->box && gc.wide == h->wide && gc.surr_mode == h->surr_mode &&
                       gc.tile == tile_code(h->sg);
    if (!match) {
        if (gc.exec) { cudaGraphExecDestroy(gc.exec); gc.exec = nullptr; }
        if (h->tiled) {   // kernel attributes are set outside the capture
            tiled_cfg<D, R>(h, 0);
            tiled_cfg<D, R>(h, 1);
        }
        const int64_t l0 = h->launches, s0 = h->steps_done, q0 = h->sorts_done;
        cudaGraph_t graph = nullptr;
        CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
        Launcher L{h};
        try {
            for (int k = 0; k < 2 * S; ++k) issue_step<D, R>(h, L, dt, Ti, Ti + dt);
        } catch (...) {
            cudaStreamEndCapture(h->stream, &graph);
            if (graph) cudaGraphDestroy(graph);
            throw;
        }
        CK(cudaStreamEndCapture(h->stream, &graph));
        cudaError_t e = cudaGraphInstantiate(&gc.exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) throw Err{MPM_E_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e)};
        gc.dt = dt;
        gc.pbuf0 = h->pbuf[0];
        gc.sort_every = S;
        gc.tiled = h->tiled;
        gc.box = h->box;
        gc.wide = h->wide;
        gc.surr_mode = h->surr_mode;
        gc.tile = tile_code(h->sg);
        gc.launches = h->launches - l0;
        gc.steps = h->steps_done - s0;
        gc.sorts = h->sorts_done - q0;
        // the capture recorded the work without running it
    } else {
        h->launches += gc.launches;
        h->steps_done += gc.steps;
        h->sorts_done += gc.sorts;
    }
    CK(cudaGraphLaunch(gc.exec, h->stream));
    h->graph_launches++;
    return true;
}

template <int D, typename R> void run_steps(mpm_handle *h, double dt, double Ti0, int64_t nsteps) {
    Launcher L{h};
    auto next_t = [&](double t) {
        return h->d.time_f32 ? (double)((float)t + (float)dt) : t + dt;
    };
    // The nodal mass, momentum and force left by the last fused pass are the
    // P2G of the current state with the gravity at acc_Ti, the only input of
    // P2G that depends on time; they are redone when the caller's Ti gives
    // another gravity (during the ramp Ti < Te).
    if (!h->acc_valid || gravity_at(h->d, h->acc_Ti) != gravity_at(h->d, Ti0)) {
        if (h->since_sort >= h->sort_every) do_sort<D, R>(h);
        standalone_p2g<D, R>(h, Ti0, L);
    }
    double Ti = Ti0;
    const int64_t block = 2 * (int64_t)h->sort_every;
    for (int64_t s = 0; s < nsteps;) {
        // (logging mode draws a new sample of particles every step: no replay)
        if (h->use_graphs && !h->profiling && h->surr_mode != 1 && Ti >= h->d.Te && h->since_sort >= h->sort_every &&
            nsteps - s >= block) {
            graph_block<D, R>(h, dt, Ti);
            for (int64_t k = 0; k < block; ++k) Ti = next_t(Ti);
            s += block;
            continue;
        }
        double Tn = next_t(Ti);
        issue_step<D, R>(h, L, dt, Ti, Tn);
        Ti = Tn;
        ++s;
    }
    h->acc_valid = true;
    h->acc_Ti = Ti;
}

// ---- dispatch helpers ----------------------------------------------------------------
template <template <int, typename> class F, typename... A> void dispatch(mpm_handle *h, A &&...a) {
    if (h->d.dim == 2) {
        if (h->fp64) F<2, double>::go(h, a...);
        else F<2, float>::go(h, a...);
    } else {
        if (h->fp64) F<3, double>::go(h, a...);
        else F<3, float>::go(h, a...);
    }
}

template <int D, typename R> struct RunSteps {
    static void go(mpm_handle *h, double dt, double Ti0, int64_t n) { run_steps<D, R>(h, dt, Ti0, n); }
};
template <int D, typename R> struct DoSort {
    static void go(mpm_handle *h) { do_sort<D, R>(h); }
};

template <int D, typename R> struct Upload {
    static void go(mpm_handle *h, const mpm_host_views *v) {
        const int64_t np = h->d.np;
        PDev<D, R> P = pdev_from<D, R>(h, 0);
        constexpr int NV = PDev<D, R>::NV, NF = PDev<D, R>::NF;
        auto req = [&](const mpm_view &vw, const char *name) {
            if (!vw.ptr) throw Err{MPM_E_ARG, std::string("missing host array ") + name};
            if (vw.ld < np) throw Err{MPM_E_ARG, std::string("leading dimension too small for ") + name};
        };
        req(v->xi, "xi");
        req(v->vs, "vs");
        req(v->sig, "sig");
        req(v->F, "F");
        req(v->Omega0, "Omega0");
        req(v->Omega, "Omega");
        req(v->rho, "rho");
        req(v->nid, "nid");
        // Materials that differ only in cohesion (the reference's way of
        // giving every particle its own random-field cohesion: nid = 1:np,
        // property.jl:62-63) are stored as one record plus a per-particle c.
        h->coh_mode = false;
        if (h->d.nmat > 1 && v->c.ptr) {
            bool same = true;
            const mpm_view *others[] = {&v->Ks, &v->Gs, &v->phi, &v->psi, &v->sigt, &v->Hp, &v->cr};
            for (const mpm_view *o : others) {
                if (!o->ptr) continue;
                const double a0 = view_get(*o, 0, 0);
                for (int64_t k = 1; k < h->d.nmat && same; ++k) same = view_get(*o, k, 0) == a0;
            }
            h->coh_mode = same;
        }
        P = pdev_from<D, R>(h, 0);
        // host arrays handed to asynchronous copies outlive them: the guard,
        // declared after them, synchronises the stream before they are freed,
        // on the error paths too
        // (left uninitialised: the parallel loops below write every entry, so
        // their pages are first touched by the threads that fill them)
        const int64_t ni = h->ni, nny = h->d.nny;
        using T4 = typename Vec<R>::T4;
        std::unique_ptr<uint32_t[]> mid(new uint32_t[np]);
        std::unique_ptr<R[]> coh;
        std::unique_ptr<uint8_t[]> mask(new uint8_t[ni]);
        std::unique_ptr<T4[]> val(new T4[ni]);
        std::unique_ptr<T4[]> valw(h->ts ? new T4[ni] : nullptr);
        std::vector<Mat<R>> M;
        StreamGuard guard{h->stream};
        if (np) {
            for (int d = 0; d < D; ++d) upload_col<double>(h, v->xi, d, P.x[d], np);
            for (int d = 0; d < D; ++d) upload_col<R>(h, v->vs, d, P.v[d], np);
            for (int c = 0; c < NV; ++c) upload_col<R>(h, v->sig, c, P.sig[c], np);
            for (int c = 0; c < NF; ++c) upload_col<R>(h, v->F, c, P.F[c], np);
            for (int c = 0; c < NV; ++c) {
                if (v->eps.ptr) upload_col<R>(h, v->eps, c, P.eps[c], np);
                else CK(cudaMemsetAsync(P.eps[c], 0, np * sizeof(R), h->stream));
            }
            auto opt = [&](const mpm_view &vw, R *dst) {
                if (vw.ptr) upload_col<R>(h, vw, 0, dst, np);
                else CK(cudaMemsetAsync(dst, 0, np * sizeof(R), h->stream));
            };
            opt(v->epsq, P.epsq);
            opt(v->epsk, P.epsk);
            opt(v->epsv, P.epsv);
            upload_col<R>(h, v->Omega0, 0, P.vol0, np);
            // particle mass ms = Ω·ρs (resetmpstatus_OS!, utils_OS.jl:199), kept per particle:
            // Ω·ρs = (J Ω0)(ρs0 / J) is invariant through the run.  Ω and ρs are staged
            // in FP64 behind the staging slot and multiplied on the device.
            double *om = (double *)(stage_area(h, np * 24) + np * 8), *rh = om + np;
            const int64_t nb = cdiv(np, 256);
            upload_col<double>(h, v->Omega, 0, om, np);
            k_convert<double, R><<<nb, 256, 0, h->stream>>>(om, P.vol, np);
            upload_col<double>(h, v->rho, 0, rh, np);
            k_mass<R><<<nb, 256, 0, h->stream>>>(om, rh, P.m, np);
            LAUNCH_CHECK();
            if (h->ts) {
                // two-phase fields (particle.jl:103-128); mw = Ω·ρw is invariant like ms
                req(v->n, "n");
                req(v->rhow, "rhow");
                if (!v->Kw.ptr || !v->kperm.ptr) throw Err{MPM_E_ARG, "two-phase model needs the Kw and k arrays"};
                int badn = 0;
#pragma omp parallel for schedule(static) reduction(| : badn)
                for (int64_t i = 0; i < np; ++i) {
                    const double n = view_get(v->n, i, 0);
                    if (!(n > 0.0 && n < 1.0)) badn = 1;
                }
                if (badn) throw Err{MPM_E_ARG, "two-phase porosity n must lie in (0, 1)"};
                upload_col<R>(h, v->n, 0, P.n, np);
                opt(v->sigw, P.sigw);
                for (int d = 0; d < D; ++d) {
                    if (v->vw.ptr) upload_col<R>(h, v->vw, d, P.vw[d], np);
                    else CK(cudaMemsetAsync(P.vw[d], 0, np * sizeof(R), h->stream));
                }
                for (int c = 0; c < NV; ++c) {
                    if (v->epsw.ptr) upload_col<R>(h, v->epsw, c, P.epsw[c], np);
                    else CK(cudaMemsetAsync(P.epsw[c], 0, np * sizeof(R), h->stream));
                }
                upload_col<double>(h, v->rhow, 0, rh, np);
                k_mass<R><<<nb, 256, 0, h->stream>>>(om, rh, P.mw, np);
                LAUNCH_CHECK();
            }
            // host-side conversions run while the column copies above are in flight;
            // their (pageable) copies are enqueued after the boundary loop
            int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
            for (int64_t i = 0; i < np; ++i) {
                const int64_t q = view_geti(v->nid, i);
                if (q < 1 || q > h->d.nmat) bad = 1;
                mid[i] = (uint32_t)(q - 1);
            }
            if (bad) throw Err{MPM_E_ARG, "nid out of range 1..nmat"};
            if (h->coh_mode) {
                // one shared material record; the cohesion travels with the particle
                coh.reset(new R[np]);
#pragma omp parallel for schedule(static)
                for (int64_t i = 0; i < np; ++i) {
                    coh[i] = (R)view_get(v->c, mid[i], 0);
                    mid[i] = 0u;
                }
            }
            k_iota<<<cdiv(np, 256), 256, 0, h->stream>>>(P.orig, np);
            LAUNCH_CHECK();
        }
        // boundary: per node in the reference's node order -> internal order
        bool anyval = false;
        const mpm_view *idx[3] = {&v->vx_idx, &v->vy_idx, &v->vz_idx};
        const mpm_view *vv[3] = {&v->vx_val, &v->vy_val, &v->vz_val};
        // water velocity BC (VBoundary *_w_*): arrays shorter than ni (the
        // reference's [0] default) mean none
        const mpm_view *widx[3] = {&v->vxw_idx, &v->vyw_idx, &v->vzw_idx};
        const mpm_view *wv[3] = {&v->vxw_val, &v->vyw_val, &v->vzw_val};
        bool anyw = false;
        const bool ts = h->ts;
#pragma omp parallel for schedule(static) reduction(|| : anyval, anyw)
        for (int64_t r = 0; r < ni; ++r) {
            int64_t inode = r;
            if (D == 2) {  // reference 2D: y descending inside a column
                int64_t ix = r / nny, rr = r % nny;
                inode = ix * nny + (nny - 1 - rr);
            }
            R vals[3] = {0, 0, 0};
            uint8_t mk = 0;
            for (int d = 0; d < D; ++d) {
                if (idx[d]->ptr && view_geti(*idx[d], r) != 0) {
                    mk |= (uint8_t)(1 << d);
                    vals[d] = vv[d]->ptr ? (R)view_get(*vv[d], r, 0) : R(0);
                    if (vals[d] != R(0)) anyval = true;
                }
            }
            if (ts) {
                R wvals[3] = {0, 0, 0};
                for (int d = 0; d < D; ++d) {
                    if (widx[d]->ptr && widx[d]->ld >= ni && view_geti(*widx[d], r) != 0) {
                        mk |= (uint8_t)(8 << d);
                        wvals[d] = (wv[d]->ptr && wv[d]->ld >= ni) ? (R)view_get(*wv[d], r, 0) : R(0);
                        if (wvals[d] != R(0)) anyw = true;
                    }
                }
                valw[inode].x = wvals[0]; valw[inode].y = wvals[1]; valw[inode].z = wvals[2]; valw[inode].w = 0;
            }
            mask[inode] = mk;
            val[inode].x = vals[0]; val[inode].y = vals[1]; val[inode].z = vals[2]; val[inode].w = 0;
        }
        if (np) {
            if (coh) CK(cudaMemcpyAsync(P.coh, coh.get(), np * sizeof(R), cudaMemcpyHostToDevice, h->stream));
            CK(cudaMemcpyAsync(P.mat, mid.get(), np * 4, cudaMemcpyHostToDevice, h->stream));
        }
        build_materials<R>(h, v, M);
        if (anyw) {
            if (!h->bcvalw) h->bcvalw = dalloc(h, ni * sizeof(T4));
            CK(cudaMemcpyAsync(h->bcvalw, valw.get(), ni * sizeof(T4), cudaMemcpyHostToDevice, h->stream));
        } else {
            h->bcvalw = nullptr;
        }
        CK(cudaMemcpyAsync(h->bcmask, mask.get(), ni, cudaMemcpyHostToDevice, h->stream));
        if (anyval) {
            if (!h->bcval) h->bcval = dalloc(h, ni * sizeof(T4));
            CK(cudaMemcpyAsync(h->bcval, val.get(), ni * sizeof(T4), cudaMemcpyHostToDevice, h->stream));
        } else {
            h->bcval = nullptr;
        }
        CK(cudaStreamSynchronize(h->stream));
        h->uploaded = true;
        h->acc_valid = false;
        h->since_sort = 1 << 30;
    }
};

template <int D, typename R> struct Download {
    static void go(mpm_handle *h, const mpm_host_views *v, uint32_t mask) {
        const int64_t np = h->d.np;
        if (!np) return;
        PDev<D, R> P = pdev_from<D, R>(h, 0);
        StreamGuard guard{h->stream};   // no copy into the caller's arrays outlives the call
        constexpr int NV = PDev<D, R>::NV, NF = PDev<D, R>::NF;
        auto chk = [&](const mpm_view &vw, const char *name) {
            if (!vw.ptr) throw Err{MPM_E_ARG, std::string("missing host array for download: ") + name};
            if (vw.ld < np) throw Err{MPM_E_ARG, std::string("leading dimension too small for ") + name};
        };
        if (mask & MPM_F_XI) { chk(v->xi, "xi"); for (int d = 0; d < D; ++d) download_col<double>(h, P.x[d], P.orig, v->xi, d, np); }
        if (mask & MPM_F_VS) { chk(v->vs, "vs"); for (int d = 0; d < D; ++d) download_col<R>(h, P.v[d], P.orig, v->vs, d, np); }
        if (mask & MPM_F_SIG) { chk(v->sig, "sig"); for (int c = 0; c < NV; ++c) download_col<R>(h, P.sig[c], P.orig, v->sig, c, np); }
        if (mask & MPM_F_EPS) { chk(v->eps, "eps"); for (int c = 0; c < NV; ++c) download_col<R>(h, P.eps[c], P.orig, v->eps, c, np); }
        if (mask & MPM_F_F) { chk(v->F, "F"); for (int c = 0; c < NF; ++c) download_col<R>(h, P.F[c], P.orig, v->F, c, np); }
        if (mask & MPM_F_EPSQ) { chk(v->epsq, "epsq"); download_col<R>(h, P.epsq, P.orig, v->epsq, 0, np); }
        if (mask & MPM_F_EPSK) { chk(v->epsk, "epsk"); download_col<R>(h, P.epsk, P.orig, v->epsk, 0, np); }
        if (mask & MPM_F_EPSV) { chk(v->epsv, "epsv"); download_col<R>(h, P.epsv, P.orig, v->epsv, 0, np); }
        if (mask & MPM_F_MS) { chk(v->ms, "ms"); download_col<R>(h, P.m, P.orig, v->ms, 0, np); }
        const uint32_t tsmask = MPM_F_MW | MPM_F_VW | MPM_F_SIGW | MPM_F_EPSW | MPM_F_N | MPM_F_RHOW;
        if ((mask & tsmask) && !h->ts) throw Err{MPM_E_ARG, "two-phase fields requested from a one-phase model"};
        if (mask & MPM_F_MW) { chk(v->mw, "mw"); download_col<R>(h, P.mw, P.orig, v->mw, 0, np); }
        if (mask & MPM_F_N) { chk(v->n, "n"); download_col<R>(h, P.n, P.orig, v->n, 0, np); }
        if (mask & MPM_F_SIGW) { chk(v->sigw, "sigw"); download_col<R>(h, P.sigw, P.orig, v->sigw, 0, np); }
        if (mask & MPM_F_VW) { chk(v->vw, "vw"); for (int d = 0; d < D; ++d) download_col<R>(h, P.vw[d], P.orig, v->vw, d, np); }
        if (mask & MPM_F_EPSW) { chk(v->epsw, "epsw"); for (int c = 0; c < NV; ++c) download_col<R>(h, P.epsw[c], P.orig, v->epsw, c, np); }
        // derived fields: k_derived writes them in original order straight into
        // the staging area; FP32 views take a converted copy behind it
        auto derived = [&](int what, const mpm_view &vw, const char *name) {
            chk(vw, name);
            double *st = (double *)stage_area(h, np * 12);
            const int64_t nb = cdiv(np, 256);
            k_derived<D, R><<<nb, 256, 0, h->stream>>>(P, np, what, st);
            LAUNCH_CHECK();
            if (vw.type == MPM_T_F64) {
                CK(cudaMemcpyAsync(vw.ptr, st, np * 8, cudaMemcpyDeviceToHost, h->stream));
            } else if (vw.type == MPM_T_F32) {
                float *f = (float *)(st + np);
                k_convert<double, float><<<nb, 256, 0, h->stream>>>(st, f, np);
                LAUNCH_CHECK();
                CK(cudaMemcpyAsync(vw.ptr, f, np * 4, cudaMemcpyDeviceToHost, h->stream));
            } else {
                throw Err{MPM_E_ARG, "float field requested into an integer view"};
            }
        };
        if (mask & MPM_F_OMEGA) derived(0, v->Omega, "Omega");
        if (mask & MPM_F_SIGM) derived(1, v->sigm, "sigm");
        if (mask & MPM_F_RHO) derived(2, v->rho, "rho");
        if (mask & MPM_F_RHOW) derived(3, v->rhow, "rhow");
        if (mask & MPM_F_P2C) {
            chk(v->p2c, "p2c");
            if (v->p2c.type != MPM_T_I64 && v->p2c.type != MPM_T_I32) throw Err{MPM_E_ARG, "p2c view must be integer"};
            int64_t *tmp = (int64_t *)stage_area(h, np * 8);
            GDev<R> g = gdev_from<R>(h);
            k_p2c<D, R><<<cdiv(np, 256), 256, 0, h->stream>>>(P, g, np, tmp);
            LAUNCH_CHECK();
            std::vector<int64_t> hv(np);
            CK(cudaMemcpyAsync(hv.data(), tmp, np * 8, cudaMemcpyDeviceToHost, h->stream));
            CK(cudaStreamSynchronize(h->stream));
            for (int64_t i = 0; i < np; ++i) {
                if (v->p2c.type == MPM_T_I64) ((int64_t *)v->p2c.ptr)[i] = hv[i];
                else ((int32_t *)v->p2c.ptr)[i] = (int32_t)hv[i];
            }
        }
        CK(cudaStreamSynchronize(h->stream));
    }
};

// ---- snapshots: the particle fields of one HDF5 group of submit_work! ------------
// (src/solver.jl:60-70: stress, strain_s, eqstrain, ekstrain, eqrate, coords,
// velocity_s, volume, mass_s), gathered into the original particle order.
struct SnapField {
    uint32_t bit;
    const char *name;
};
constexpr SnapField kSnapFields[] = {
    {MPM_F_SIG, "stress"},    {MPM_F_EPS, "strain_s"},   {MPM_F_EPSQ, "eqstrain"},
    {MPM_F_EPSK, "ekstrain"}, {MPM_F_EPSV, "eqrate"},    {MPM_F_XI, "coords"},
    {MPM_F_VS, "velocity_s"}, {MPM_F_OMEGA, "volume"},   {MPM_F_MS, "mass_s"},
    // two-phase groups (src/solver.jl:73-76)
    {MPM_F_SIGW, "pressure_w"}, {MPM_F_EPSW, "strain_w"}, {MPM_F_VW, "velocity_w"}, {MPM_F_N, "porosity"}};

int snap_columns(uint32_t bit, int dim) {
    const int nv = dim == 2 ? 4 : 6;
    switch (bit) {
    case MPM_F_SIG: case MPM_F_EPS: case MPM_F_EPSW: return nv;
    case MPM_F_XI: case MPM_F_VS: case MPM_F_VW: return dim;
    default: return 1;
    }
}

struct SnapCols {
    const void *src[40];
    int32_t f64[40];   // 1: the column is FP64 (positions), else the bulk type
};

template <typename R, typename O>
__global__ void k_snap_gather(SnapCols c, const uint32_t *orig, int64_t np, O *out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    const int col = blockIdx.y;
    const double v = c.f64[col] ? ((const double *)c.src[col])[i] : (double)((const R *)c.src[col])[i];
    out[(int64_t)col * np + orig[i]] = (O)v;
}

template <int D, typename R> struct SnapGather {
    // Launches the gather of `mask`'s fields into `out` (element type `type`) on the compute stream.
    static void go(mpm_handle *h, uint32_t mask, int32_t type, void *out) {
        const int64_t np = h->d.np;
        PDev<D, R> P = pdev_from<D, R>(h, 0);
        constexpr int NV = PDev<D, R>::NV;
        SnapCols c{};
        int n = 0;
        auto add = [&](const void *p, int f64) { c.src[n] = p; c.f64[n] = f64; ++n; };
        for (const SnapField &f : kSnapFields) {
            if (!(mask & f.bit)) continue;
            switch (f.bit) {
            case MPM_F_SIG: for (int k = 0; k < NV; ++k) add(P.sig[k], 0); break;
            case MPM_F_EPS: for (int k = 0; k < NV; ++k) add(P.eps[k], 0); break;
            case MPM_F_EPSQ: add(P.epsq, 0); break;
            case MPM_F_EPSK: add(P.epsk, 0); break;
            case MPM_F_EPSV: add(P.epsv, 0); break;
            case MPM_F_XI: for (int d = 0; d < D; ++d) add(P.x[d], 1); break;
            case MPM_F_VS: for (int d = 0; d < D; ++d) add(P.v[d], 0); break;
            case MPM_F_OMEGA: add(P.vol, 0); break;
            case MPM_F_MS: add(P.m, 0); break;
            case MPM_F_SIGW: add(P.sigw, 0); break;
            case MPM_F_EPSW: for (int k = 0; k < NV; ++k) add(P.epsw[k], 0); break;
            case MPM_F_VW: for (int d = 0; d < D; ++d) add(P.vw[d], 0); break;
            case MPM_F_N: add(P.n, 0); break;
            }
        }
        if (!n || !np) return;
        const dim3 grid((unsigned)cdiv(np, 256), (unsigned)n);
        if (type == MPM_T_F64) k_snap_gather<R, double><<<grid, 256, 0, h->stream>>>(c, P.orig, np, (double *)out);
        else k_snap_gather<R, float><<<grid, 256, 0, h->stream>>>(c, P.orig, np, (float *)out);
        LAUNCH_CHECK();
        ++h->launches;
    }
};

template <int D, typename R> struct P2CAll {
    static void go(mpm_handle *h, int64_t *out) {
        const int64_t np = h->d.np;
        if (!np) return;
        PDev<D, R> P = pdev_from<D, R>(h, 0);
        GDev<R> g = gdev_from<R>(h);
        int64_t *tmp = (int64_t *)stage_area(h, np * 8);
        k_p2c<D, R><<<cdiv(np, 256), 256, 0, h->stream>>>(P, g, np, tmp);
        LAUNCH_CHECK();
        CK(cudaMemcpyAsync(out, tmp, np * 8, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    }
};

template <typename R>
__global__ void k_count_active(const Node8<R> *acc, int64_t ni, unsigned long long *out) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long c = (i < ni && acc[i].a.x > 0) ? 1ull : 0ull;
    c = __reduce_add_sync(0xffffffffu, (unsigned)c);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}

template <int D, typename R> struct CountActive {
    static void go(mpm_handle *h, int64_t *out) {
        using T4 = typename Vec<R>::T4;
        unsigned long long *d = (unsigned long long *)h->bsum;   // scratch word
        CK(cudaMemsetAsync(d, 0, 8, h->stream));
        k_count_active<R><<<cdiv(h->ni, 256), 256, 0, h->stream>>>((const Node8<R> *)h->acc, h->ni, d);
        LAUNCH_CHECK();
        unsigned long long v = 0;
        CK(cudaMemcpyAsync(&v, d, 8, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        *out = (int64_t)v;
    }
};

template <int D, typename R> struct Order {
    static void go(mpm_handle *h, int64_t *out) {
        const int64_t np = h->d.np;
        if (!np) return;
        PDev<D, R> P = pdev_from<D, R>(h, 0);
        std::vector<uint32_t> o(np);
        CK(cudaMemcpyAsync(o.data(), P.orig, np * 4, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        for (int64_t i = 0; i < np; ++i) out[i] = o[i];
    }
};

template <int D, typename R> struct Stages {
    static void go(mpm_handle *h, double dt, double Ti, uint32_t mask) {
        const int64_t np = h->d.np;
        Launcher L{h};
        const int nblk = h->nbx * h->nby * h->nbz;
        const int ngrid = std::min(nblk, h->nsm * 16);
        if (mask & 1u) standalone_p2g<D, R>(h, Ti, L);
        PDev<D, R> P = pdev_from<D, R>(h, 0);
        GDev<R> g = gdev_from<R>(h);
        StepParams sp = make_params<D, R>(h, dt, Ti, gravity_at(h->d, Ti));
        if (mask & 2u) L.run("solve", [&] { k_solve<D, R><<<ngrid, Blk<D>::NT, 0, h->stream>>>(g, sp); });
        if ((mask & 4u) && np) L.run("dmap", [&] { k_dmap<D, R><<<cdiv(np, 256), 256, 0, h->stream>>>(P, g, sp); });
        if (mask & 8u) {
            L.run("dm3", [&] { k_dm3<D, R><<<ngrid, Blk<D>::NT, 0, h->stream>>>(g, sp); });
            CK(cudaMemsetAsync(h->bcount, 0, 4, h->stream));
        }
        const bool mc3 = sp.mc3d && sp.constitutive == MPM_MOHRCOULOMB;
        if ((mask & 16u) && np) L.run("g2p", [&] {
            if (mc3) k_g2p<D, R, false, D == 3><<<cdiv(np, 256), 256, g2p_smem(sp), h->stream>>>(P, g, sp);
            else k_g2p<D, R, false><<<cdiv(np, 256), 256, g2p_smem(sp), h->stream>>>(P, g, sp);
        });
        h->acc_valid = false;
    }
};

template <int D, typename R> struct GridOut {
    static void go(mpm_handle *h, int field, double *out) {
        using T4 = typename Vec<R>::T4;
        const int64_t ni = h->ni, nny = h->d.nny;
        std::vector<T4> a(ni);
        // field -> (record array, half): 0 mass, 1 momentum (acc.a), 2 force (acc.b),
        // 3 vsT (gat.a), 4 as / 5 Δus (gat.b: as after the solve, Δus after DM3), 6 vs
        if (field < 0 || field > 6) throw Err{MPM_E_ARG, "grid field out of range"};
        if (field == 6) {
            if (!h->gvs) throw Err{MPM_E_ARG, "grid vs is kept only with PIC != 0 or va = :v"};
            CK(cudaMemcpy(a.data(), h->gvs, ni * sizeof(T4), cudaMemcpyDeviceToHost));
        } else {
            std::vector<Node8<R>> rec(ni);
            CK(cudaMemcpy(rec.data(), field <= 2 ? h->acc : h->gat, ni * sizeof(Node8<R>), cudaMemcpyDeviceToHost));
            const bool second = field == 2 || field == 4 || field == 5;
            for (int64_t r = 0; r < ni; ++r) a[r] = second ? rec[r].b : rec[r].a;
        }
        for (int64_t r = 0; r < ni; ++r) {
            int64_t inode = r;
            if (D == 2) {
                int64_t ix = r / nny, rr = r % nny;
                inode = ix * nny + (nny - 1 - rr);
            }
            const T4 &q = a[inode];
            if (field == 0) { out[r] = (double)q.x; continue; }
            double c[3];
            if (field == 1) { c[0] = q.y; c[1] = q.z; c[2] = q.w; }
            else { c[0] = q.x; c[1] = q.y; c[2] = q.z; }
            for (int d = 0; d < D; ++d) out[r + ni * d] = c[d];
        }
    }
};

// Writer thread of a handle's snapshots: waits for each slot's device-to-host
// copy, writes the slot's fields as group<i>/<name> and group<i>/time, frees
// the slot.  Ends when asked to stop and the queue is empty.
void snap_writer(SnapState *S) {
    cudaSetDevice(S->device);
    std::unique_lock<std::mutex> lk(S->mu);
    while (true) {
        S->cv.wait(lk, [&] { return S->stop || !S->q.empty(); });
        if (S->q.empty()) break;
        const SnapJob j = S->q.front();
        lk.unlock();
        int rc = MPM_OK;
        std::string msg;
        const cudaError_t e = cudaEventSynchronize(S->copied[j.slot]);
        if (e != cudaSuccess) {
            rc = MPM_E_CUDA;
            msg = std::string("snapshot copy: ") + cudaGetErrorString(e);
        }
        const size_t es = j.type == MPM_T_F64 ? 8 : 4;
        const char *base = (const char *)S->host[j.slot];
        const std::string g = "group" + std::to_string(j.group) + "/";
        for (const SnapField &f : kSnapFields) {
            if (rc != MPM_OK) break;
            if (!(j.mask & f.bit)) continue;
            const int k = snap_columns(f.bit, S->dim);
            const int64_t dims[2] = {k, S->np};   // a Julia np x k matrix is the dataspace (k, np)
            rc = mpm_h5_write(j.file, (g + f.name).c_str(), j.type, k > 1 ? 2 : 1, k > 1 ? dims : dims + 1, base);
            if (rc != MPM_OK) msg = mpm_last_error(nullptr);
            base += (size_t)k * S->np * es;
        }
        if (rc == MPM_OK) {
            const double t64 = j.Ti;
            const float t32 = (float)j.Ti;
            rc = mpm_h5_write(j.file, (g + "time").c_str(), j.type, 0, nullptr,
                              j.type == MPM_T_F64 ? (const void *)&t64 : (const void *)&t32);
            if (rc != MPM_OK) msg = mpm_last_error(nullptr);
        }
        lk.lock();
        S->q.pop_front();
        S->busy[j.slot] = false;
        if (rc == MPM_OK) ++S->written;
        else if (S->err == MPM_OK) {
            S->err = rc;
            S->msg = msg;
        }
        S->cv.notify_all();
    }
}

void snap_destroy(mpm_handle *h) {
    SnapState *S = h->snap;
    if (!S) return;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
    }
    S->cv.notify_all();
    if (S->th.joinable()) S->th.join();
    for (int k = 0; k < 2; ++k) {
        if (S->dev[k]) cudaFree(S->dev[k]);
        if (S->host[k]) cudaFreeHost(S->host[k]);
        if (S->gathered[k]) cudaEventDestroy(S->gathered[k]);
        if (S->copied[k]) cudaEventDestroy(S->copied[k]);
    }
    if (S->copy) cudaStreamDestroy(S->copy);
    delete S;
    h->snap = nullptr;
}

int fail(mpm_handle *h, const Err &e) {
    if (h) h->last_error = e.msg;
    return e.code;
}

int check_flags(mpm_handle *h) {
    int f = 0;
    CK(cudaMemcpyAsync(&f, h->err, 4, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->err_host |= f;
    if (f & ERR_NAN) throw Err{MPM_E_NAN, "non-finite particle state"};
    if (f & ERR_J) throw Err{MPM_E_NONPOSITIVE_J, "det(F) <= 0 on some particle"};
    if (f & ERR_OOG) throw Err{MPM_E_OUT_OF_GRID, "a particle's uGIMP stencil left the grid (pad the grid by >= 2 cells)"};
    if (f & ERR_OVF) throw Err{MPM_E_CELL_OVERFLOW, "more than 4096 particles in one cell"};
    if (h->surr_err) {
        int se = 0;
        CK(cudaMemcpy(&se, h->surr_err, 4, cudaMemcpyDeviceToHost));
        if (se) throw Err{MPM_E_CUDA, "surrogate: a tensor-core completion wait timed out"};
    }
    return 0;
}

thread_local std::string g_create_error;

}  // namespace

namespace mpm_detail {
__attribute__((visibility("hidden"))) void set_global_error(const std::string &m) { g_create_error = m; }
}

// =====================================================================================
// C ABI
// =====================================================================================
extern "C" {

int mpm_create(const mpm_desc *d, mpm_handle **out) {
    if (!d || !out) return MPM_E_ARG;
    *out = nullptr;
    mpm_handle *h = new (std::nothrow) mpm_handle();
    if (!h) return MPM_E_ARG;
    try {
        if (d->abi_version != MPM_ABI_VERSION) throw Err{MPM_E_ARG, "ABI version mismatch"};
        if (d->dim != 2 && d->dim != 3) throw Err{MPM_E_ARG, "dim must be 2 or 3"};
        if (d->np < 0 || d->np >= (int64_t)UINT32_MAX) throw Err{MPM_E_ARG, "np out of range"};
        if (d->nmat < 1) throw Err{MPM_E_ARG, "need at least one material"};
        int64_t nnz = d->dim == 3 ? d->nnz : 1;
        if (d->nnx < 4 || d->nny < 4 || (d->dim == 3 && d->nnz < 4)) throw Err{MPM_E_ARG, "grid needs >= 4 nodes per axis"};
        int64_t ni = d->nnx * d->nny * nnz;
        if (ni >= (int64_t)1 << 31) throw Err{MPM_E_ARG, "grid larger than 2^31 nodes"};
        if (!(d->dx > 0 && d->dy > 0 && (d->dim == 2 || d->dz > 0))) throw Err{MPM_E_ARG, "cell size must be positive"};
        if (!(d->lpx > 0 && d->lpx <= d->dx && d->lpy > 0 && d->lpy <= d->dy &&
              (d->dim == 2 || (d->lpz > 0 && d->lpz <= d->dz))))
            throw Err{MPM_E_ARG, "particle size must satisfy 0 < lp <= h (at most 3 uGIMP nodes per axis)"};
        if (d->constitutive < 0 || d->constitutive > 2) throw Err{MPM_E_UNSUPPORTED, "constitutive model not provided (hyperelastic is out of scope)"};
        if (d->mc3d != MPM_MC3D_LITERAL && d->mc3d != MPM_MC3D_RESTATED) throw Err{MPM_E_ARG, "mc3d must be 0 or 1"};
        if (d->scheme != MPM_SCHEME_MUSL && d->scheme != MPM_SCHEME_USL) throw Err{MPM_E_ARG, "scheme must be 0 (MUSL) or 1 (USL)"};
        if (d->coupling != MPM_COUPLING_OS && d->coupling != MPM_COUPLING_TS) throw Err{MPM_E_ARG, "coupling must be 0 (OS) or 1 (TS)"};
        if (d->coupling == MPM_COUPLING_TS && d->scheme != MPM_SCHEME_MUSL)
            throw Err{MPM_E_UNSUPPORTED, "the two-phase coupling has the MUSL scheme only (TS_MUSL.jl)"};
        if (d->coupling == MPM_COUPLING_TS && d->mvl)
            throw Err{MPM_E_UNSUPPORTED, "MVL with the two-phase coupling is not provided"};
        h->d = *d;
        h->ts = d->coupling == MPM_COUPLING_TS;
        if (h->d.dim == 2) { h->d.nnz = 1; h->d.z1 = 0; h->d.dz = 1; h->d.lpz = 1; }
        h->fp64 = d->precision == MPM_PREC_FP64;
        // re-sort period: particles move far less than a cell per step (CFL 0.2
        // on the wave speed); with the lane merging 32 steps measured 1-2 %
        // faster than 16 on the column, slope and saturated-column workloads
        h->sort_every = d->sort_every > 0 ? d->sort_every : 32;
        h->ni = ni;
        CK(cudaSetDevice(d->device));
        h->dev = d->device;
        CK(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
        CK(cudaEventCreate(&h->ev0));
        CK(cudaEventCreate(&h->ev1));
        const size_t R = h->fp64 ? 8 : 4;
        const size_t T4 = 4 * R;
        size_t pb = pbuf_bytes(d->dim, h->fp64, d->np, h->ts);
        h->pbuf[0] = dalloc(h, pb);
        h->pbuf[1] = dalloc(h, pb);
        h->pbuf_size = pb;
        h->acc = dalloc(h, ni * 2 * T4);
        h->gat = dalloc(h, ni * 2 * T4);
        h->gvs = (d->PIC != 0.0 || d->va == MPM_VA_V) ? dalloc(h, ni * T4) : nullptr;
        CK(cudaMemset(h->acc, 0, ni * 2 * T4));
        CK(cudaMemset(h->gat, 0, ni * 2 * T4));
        if (h->ts) {
            h->accw = dalloc(h, ni * 2 * T4);
            h->accd = dalloc(h, ni * T4);
            h->gatw = dalloc(h, ni * 2 * T4);
            CK(cudaMemset(h->accw, 0, ni * 2 * T4));
            CK(cudaMemset(h->accd, 0, ni * T4));
            CK(cudaMemset(h->gatw, 0, ni * 2 * T4));
        }
        if (h->gvs) CK(cudaMemset(h->gvs, 0, ni * T4));
        h->bcmask = (uint8_t *)dalloc(h, ni);
        CK(cudaMemset(h->bcmask, 0, ni));
        if (d->dim == 3) {
            h->nbx = (int)cdiv(d->nnx, Blk<3>::BX); h->nby = (int)cdiv(d->nny, Blk<3>::BY); h->nbz = (int)cdiv(nnz, Blk<3>::BZ);
        } else {
            h->nbx = (int)cdiv(d->nnx, Blk<2>::BX); h->nby = (int)cdiv(d->nny, Blk<2>::BY); h->nbz = 1;
        }
        size_t nblk = (size_t)h->nbx * h->nby * h->nbz;
        h->bflag = (uint32_t *)dalloc(h, nblk * 4);
        CK(cudaMemset(h->bflag, 0, nblk * 4));
        if (d->mvl) {
            h->nc = (d->nnx - 1) * (d->nny - 1) * (d->dim == 3 ? (d->nnz - 1) : 1);
            const size_t rs = h->fp64 ? 8 : 4;
            h->csigm = dalloc(h, (size_t)h->nc * rs);
            h->comega = dalloc(h, (size_t)h->nc * rs);
            h->pcell = (uint32_t *)dalloc(h, (size_t)std::max<int64_t>(d->np, 1) * 4);
        }
        h->blist = (uint32_t *)dalloc(h, nblk * 4);
        h->bcount = (uint32_t *)dalloc(h, 4);
        CK(cudaMemset(h->bcount, 0, 4));
        size_t msz = h->fp64 ? sizeof(Mat<double>) : sizeof(Mat<float>);
        h->mat = dalloc(h, d->nmat * msz);
        h->err = (int *)dalloc(h, 4);
        CK(cudaMemset(h->err, 0, 4));
        // sort geometry: tiles of 32 cells by default (MPM_B200_TILE=AxBxC picks
        // another shape: 32, 64 or 128 cells)
        SortGeom &sg = h->sg;
        int tsh[3] = {d->dim == 3 ? Tile<3>::TX : Tile<2>::TX, d->dim == 3 ? Tile<3>::TY : Tile<2>::TY,
                      d->dim == 3 ? Tile<3>::TZ : 1};
        if (const char *e = getenv("MPM_B200_TILE")) {
            int a = 0, b = 0, c = 1;
            if (std::sscanf(e, "%dx%dx%d", &a, &b, &c) >= 2) { tsh[0] = a; tsh[1] = b; tsh[2] = d->dim == 3 ? c : 1; }
        }
        const int cpt = tsh[0] * tsh[1] * tsh[2];
        if (tsh[0] < 1 || tsh[1] < 1 || tsh[2] < 1 || (cpt != 32 && cpt != 64 && cpt != 128))
            throw Err{MPM_E_ARG, "tile shape must hold 32, 64 or 128 cells"};
        const int64_t nk = sort_geom(sg, d->dim, d->nnx, d->nny, nnz, tsh[0], tsh[1], tsh[2]);
        // the sort buffers hold the keys of any tile shape mpm_set_tile may pick
        int64_t nk_max = nk;
        for (const TileShape &ts : tile_shapes(d->dim)) {
            SortGeom t{};
            nk_max = std::max(nk_max, sort_geom(t, d->dim, d->nnx, d->nny, nnz, ts.tx, ts.ty, ts.tz));
        }
        if (nk_max >= (int64_t)LOW29 || d->np >= (int64_t)LOW29)
            throw Err{MPM_E_ARG, "grid or particle count beyond the sort's 2^29 limit"};
        h->nk = (uint32_t)nk;
        h->nk_cap = (uint32_t)nk_max;
        int64_t npa = std::max<int64_t>(d->np, 1);
        h->keys = (uint32_t *)dalloc(h, npa * 4);
        h->cnt = (uint32_t *)dalloc(h, (size_t)h->nk_cap * 4);
        h->off = (uint32_t *)dalloc(h, ((size_t)h->nk_cap + 1) * 4);
        h->bsum = (uint32_t *)dalloc(h, (cdiv(h->nk_cap, SCAN_CHUNK) + 1) * 4);
        h->big_cap = 65536;
        h->big = (uint32_t *)dalloc(h, h->big_cap * 4);
        h->nbig = (uint32_t *)dalloc(h, 4);
        h->pairs = (uint2 *)dalloc(h, npa * 8);
        h->pairs2 = (uint2 *)dalloc(h, npa * 8);
        h->ntile_total = h->nk / (uint32_t)sg.cpt;
        h->tiles = (uint32_t *)dalloc(h, (size_t)(h->nk_cap / 32 + 1) * 4);
        h->ntiles = (uint32_t *)dalloc(h, 4);
        CK(cudaMemset(h->ntiles, 0, 4));
        CK(cudaDeviceGetAttribute(&h->nsm, cudaDevAttrMultiProcessorCount, d->device));
        // MPM_B200_TILED=1 selects the shared-memory tiled particle passes instead
        // of the per-particle kernels (vector reductions into L2); both compute the
        // same step.  The per-particle kernels are the faster ones on B200, where
        // shared-memory float atomics are the tiled passes' limiter.
        if (const char *e = getenv("MPM_B200_TILED")) h->tiled = (e[0] == '1');
        // MPM_B200_GRAPHS=0 issues every step's launches directly instead of
        // replaying captured blocks of steps.
        if (const char *e = getenv("MPM_B200_GRAPHS")) h->use_graphs = (e[0] != '0');
        if (const char *e = getenv("MPM_B200_PREFETCH")) h->prefetch = (e[0] != '0');
        if (const char *e = getenv("MPM_B200_ORDER")) h->cell_major = (std::string(e) == "cell");
        if (const char *e = getenv("MPM_B200_CHAIN")) h->chain = std::atoi(e) != 0;
        if (const char *e = getenv("MPM_B200_BOX")) h->box = std::atoi(e) != 0;
        // 3D models start with the fused pass at 3 resident CTAs per SM
        // (variant 3): measured faster on the 3D column and slope (0.414 ->
        // 0.400 ms, 1.267 -> 1.243 ms), slower on the 2D slope batch
        h->wide = h->d.dim == 3 && !h->box;
        h->work = (uint32_t *)dalloc(h, 16);
        if (!h->fp64) box_prepare(h);
        *out = h;
        return MPM_OK;
    } catch (const Err &e) {
        g_create_error = e.msg;
        for (void *p : h->allocs) cudaFree(p);
        if (h->stream) cudaStreamDestroy(h->stream);
        delete h;
        return e.code;
    }
}

int mpm_upload(mpm_handle *h, const mpm_host_views *v) {
    if (!h || !v) return MPM_E_ARG;
    try {
        CK(cudaSetDevice(h->dev));
        dispatch<Upload>(h, v);
        return MPM_OK;
    } catch (const Err &e) { return fail(h, e); }
}

int mpm_step_async(mpm_handle *h, double dt, double Ti0, int64_t nsteps) {
    if (!h) return MPM_E_ARG;
    try {
        if (!h->uploaded) throw Err{MPM_E_STATE, "mpm_step before mpm_upload"};
        if (!(dt > 0) || nsteps < 0) throw Err{MPM_E_ARG, "dt must be > 0 and nsteps >= 0"};
        CK(cudaSetDevice(h->dev));
        if (h->profiling) { for (auto &k : h->ktimes) { k.ms = 0; k.n = 0; } }
        CK(cudaEventRecord(h->ev0, h->stream));
        dispatch<RunSteps>(h, dt, Ti0, nsteps);
        CK(cudaEventRecord(h->ev1, h->stream));
        return MPM_OK;
    } catch (const Err &e) { return fail(h, e); }
}

int mpm_sync(mpm_handle *h) {
    if (!h) return MPM_E_ARG;
    try {
        CK(cudaSetDevice(h->dev));
        CK(cudaStreamSynchronize(h->stream));
        float ms = 0;
        if (cudaEventElapsedTime(&ms, h->ev0, h->ev1) == cudaSuccess) h->last_step_ms = ms;
        return check_flags(h);
    } catch (const Err &e) { return fail(h, e); }
}

int mpm_step(mpm_handle *h, double dt, double Ti0, int64_t nsteps, double *Ti_out) {
    int rc = mpm_step_async(h, dt, Ti0, nsteps);
    if (rc) return rc;
    rc = mpm_sync(h);
    if (Ti_out) {
        double t = Ti0;
        for (int64_t s = 0; s < nsteps; ++s) t = h->d.time_f32 ? (double)((float)t + (float)dt) : t + dt;
        *Ti_out = t;
    }
    return rc;
}

int mpm_set_surrogate(mpm_handle *h, const float *params, const float *norm, int32_t flags, float tol, float sref,
                      int32_t on) {
    if (!h) return MPM_E_ARG;
    try {
        CK(cudaSetDevice(h->dev));
        if (!on) {
            if (h->surr_mode == 2) h->surr_mode = 0;
            return MPM_OK;
        }
        if (!params || !norm || !(tol > 0) || !(sref > 0)) throw Err{MPM_E_ARG, "surrogate: params, norm, tol > 0, sref > 0"};
        const bool mc = h->d.constitutive == MPM_MOHRCOULOMB && h->d.mc3d == MPM_MC3D_RESTATED;
        if (h->d.dim != 3 || (h->d.constitutive != MPM_DRUCKERPRAGER && !mc))
            throw Err{MPM_E_UNSUPPORTED,
                      "the surrogate replaces the 3D Drucker-Prager or the restated 3D Mohr-Coulomb return"};
        if (h->d.mvl || h->d.scheme != MPM_SCHEME_MUSL)
            throw Err{MPM_E_UNSUPPORTED, "the surrogate runs with the MUSL scheme and without MVL"};
        const int64_t np = h->d.np;
        const int npar = mpm_mlp_nparams();
        if (!h->surr_params) {
            h->surr_params = (float *)dalloc(h, (size_t)npar * 4);
            h->surr_norm = (float *)dalloc(h, 64 * 4);
            h->surr_feat = (float *)dalloc(h, (size_t)std::max<int64_t>(np, 1) * 16 * 4);
            h->surr_out = (float *)dalloc(h, (size_t)std::max<int64_t>(np, 1) * 6 * 4);
            h->surr_list = (uint32_t *)dalloc(h, (size_t)std::max<int64_t>(np, 1) * 4);
            h->surr_s0 = (float *)dalloc(h, (size_t)std::max<int64_t>(np, 1) * 6 * 4);
            h->surr_cnt = (uint32_t *)dalloc(h, 4);
            h->surr_stats = (unsigned long long *)dalloc(h, 16);
            h->surr_err = (int *)dalloc(h, 4);
            CK(cudaMemset(h->surr_stats, 0, 16));
            CK(cudaMemset(h->surr_err, 0, 4));
            CK(cudaMemset(h->surr_cnt, 0, 4));
        }
        CK(cudaMemcpy(h->surr_params, params, (size_t)npar * 4, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(h->surr_norm, norm, 64 * 4, cudaMemcpyHostToDevice));
        CK(mpm_detail::mlp_forward_prepare());
        h->surr_tol = tol;
        h->surr_sref = sref;
        h->surr_residual = flags & 1;
        h->surr = mpm::SurrCtx{};
        h->surr.cap = (uint32_t)np;
        h->surr.feat = h->surr_feat;
        h->surr.cnt = h->surr_cnt;
        h->surr.list = h->surr_list;
        h->surr.tgt = mc ? h->surr_s0 : nullptr;   // Mohr-Coulomb: the deferred rows' pre-increment stress
        h->surr_mode = 2;
        return MPM_OK;
    } catch (const Err &e) { return fail(h, e); }
}

int mpm_log_samples(mpm_handle *h, float *feat, float *target, uint32_t *count, uint32_t cap, uint32_t every) {
    if (!h) return MPM_E_ARG;
    if (every == 0) {
        if (h->surr_mode == 1) { h->surr_mode = 0; h->surr = mpm::SurrCtx{}; }
        return MPM_OK;
    }
    if (!feat || !target || !count || cap == 0) {
        h->last_error = "mpm_log_samples: feat, target, count and cap > 0 are required";
        return MPM_E_ARG;
    }
    if (h->d.dim != 3 || !(h->d.constitutive == MPM_DRUCKERPRAGER ||
                           (h->d.constitutive == MPM_MOHRCOULOMB && h->d.mc3d == MPM_MC3D_RESTATED))) {
        h->last_error = "sample logging covers the 3D Drucker-Prager and the restated 3D Mohr-Coulomb return";
        return MPM_E_UNSUPPORTED;
    }
    h->surr = mpm::SurrCtx{};
    h->surr.every = every;
    h->surr.cap = cap;
    h->surr.feat = feat;
    h->surr.tgt = target;
    h->surr.cnt = count;
    h->surr_mode = 1;
    return MPM_OK;
}

int mpm_set_tuning(mpm_handle *h, int32_t sort_every, int32_t tiled) {
    if (!h) return MPM_E_ARG;
    if (sort_every < 1 || sort_every > 1024 || tiled < 0 || tiled > 3) {
        h->last_error = "sort_every must be 1..1024 and the particle-pass variant 0, 1, 2 or 3";
        return MPM_E_ARG;
    }
    h->sort_every = sort_every;
    h->tiled = tiled == 1;
    h->box = tiled == 2;
    h->wide = tiled == 3;
    return MPM_OK;
}

int mpm_get_tuning(mpm_handle *h, int32_t *sort_every, int32_t *tiled) {
    if (!h) return MPM_E_ARG;
    if (sort_every) *sort_every = h->sort_every;
    if (tiled) *tiled = h->tiled ? 1 : (h->box ? 2 : (h->wide ? 3 : 0));
    return MPM_OK;
}

int mpm_set_tile(mpm_handle *h, int32_t tx, int32_t ty, int32_t tz) {
    if (!h) return MPM_E_ARG;
    try {
        const int D = h->d.dim;
        if (D == 2) tz = 1;
        bool known = false;
        for (const TileShape &t : tile_shapes(D)) known = known || (t.tx == tx && t.ty == ty && t.tz == tz);
        if (!known) throw Err{MPM_E_ARG, "tile shape not among the compiled ones (3D: 2x8x2, 4x8x1, 4x4x2; 2D: 4x8, 2x16)"};
        SortGeom sg{};
        const int64_t nk = sort_geom(sg, D, h->d.nnx, h->d.nny, D == 3 ? h->d.nnz : 1, tx, ty, tz);
        if (nk > (int64_t)h->nk_cap) throw Err{MPM_E_STATE, "tile shape needs more sort keys than allocated"};
        h->sg = sg;
        h->nk = (uint32_t)nk;
        h->ntile_total = h->nk / (uint32_t)sg.cpt;
        h->since_sort = 1 << 30;   // the next step re-sorts with the new tiles
        return MPM_OK;
    } catch (const Err &e) { return fail(h, e); }
}

int mpm_get_tile(mpm_handle *h, int32_t *tx, int32_t *ty, int32_t *tz) {
    if (!h) return MPM_E_ARG;
    if (tx) *tx = h->sg.tx;
    if (ty) *ty = h->sg.ty;
    if (tz) *tz = h->sg.tz;
    return MPM_OK;
}

// Times every candidate on real steps of the simulation and keeps the fastest.
// Candidates, in the order of trial_ms: for each compiled tile shape (the
// default first) the re-sort periods 8, 16, 32, 64 with the default particle
// passes, then the shared-memory tiled passes and the box passes (default
// shape) at periods 16 and 32 each.  A trial runs max(steps_per_trial, period) steps starting with a
// sort, so the sort is charged once per period.  The trial steps advance the
// model like mpm_step does.  The chosen shape is reported by mpm_get_tile.
int mpm_autotune(mpm_handle *h, double dt, double Ti0, int64_t steps_per_trial, double *Ti_out,
                 int32_t *sort_every_out, int32_t *tiled_out, double *trial_ms, int32_t trial_cap) {
    static const int32_t periods[] = {8, 16, 32, 64};
    if (!h) return MPM_E_ARG;
    if (steps_per_trial < 1) {
        h->last_error = "steps_per_trial must be >= 1";
        return MPM_E_ARG;
    }
    double Ti = Ti0;
    double best = 1e300;
    int32_t best_s = h->sort_every, best_t = h->tiled ? 1 : (h->box ? 2 : (h->wide ? 3 : 0));
    TileShape best_shape{h->sg.tx, h->sg.ty, h->sg.tz};
    struct Cand { double ms = 1e300; TileShape ts{}; int32_t S = 0, t = 0; };
    Cand best0, best_other;   // fastest of variant 0, fastest of the other variants
    int k = 0;
    // one timed run of n steps (n = 0: max(steps_per_trial, S)) with the given
    // shape, period and variant, starting with a sort; returns ms per step
    auto run = [&](const TileShape &ts, int32_t S, int32_t t, int64_t n, double &ms) -> int {
        int rc = mpm_set_tile(h, ts.tx, ts.ty, ts.tz);
        if (!rc) rc = mpm_set_tuning(h, S, t);
        if (rc) return rc;
        h->since_sort = 1 << 30;
        if (n == 0) n = std::max<int64_t>(steps_per_trial, S);
        rc = mpm_step(h, dt, Ti, n, &Ti);
        if (rc) return rc;
        ms = h->last_step_ms / (double)n;
        if (trial_ms && k < trial_cap) trial_ms[k] = ms;
        ++k;
        return MPM_OK;
    };
    auto trial = [&](const TileShape &ts, int32_t S, int32_t t) -> int {
        double ms = 0;
        if (int rc = run(ts, S, t, 0, ms)) return rc;
        Cand &c = t == 0 ? best0 : best_other;
        if (ms < c.ms) c = Cand{ms, ts, S, t};
        if (ms < best) { best = ms; best_s = S; best_t = t; best_shape = ts; }
        return MPM_OK;
    };
    const std::vector<TileShape> shapes = tile_shapes(h->d.dim);
    for (const TileShape &ts : shapes)
        for (int32_t S : periods)
            if (int rc = trial(ts, S, 0)) return rc;
    // the fused pass with the other register cap, at the best shape so far
    const TileShape shape0 = best_shape;
    for (int32_t S : {32, 64})
        if (int rc = trial(shape0, S, 3)) return rc;
    for (int32_t v : {1, 2})
        for (int32_t S : {16, 32})
            if (int rc = trial(shapes[0], S, v)) return rc;
    // The trial steps advance the model, and a flow whose active region grows
    // makes later trials slower: the two finalists (the fastest variant-0
    // candidate and the fastest of the others) are timed again back to back,
    // 64 steps each, and the faster of that pair is kept.
    {
        double m0 = 0, m1 = 0;
        if (int rc = run(best0.ts, best0.S, 0, 64, m0)) return rc;
        if (int rc = run(best_other.ts, best_other.S, best_other.t, 64, m1)) return rc;
        const Cand &w = m1 < m0 ? best_other : best0;
        best_s = w.S; best_t = w.t; best_shape = w.ts;
    }
    mpm_set_tile(h, best_shape.tx, best_shape.ty, best_shape.tz);
    mpm_set_tuning(h, best_s, best_t);
    if (Ti_out) *Ti_out = Ti;
    if (sort_every_out) *sort_every_out = best_s;
    if (tiled_out) *tiled_out = best_t;
    return MPM_OK;
}

int mpm_download(mpm_handle *h, const mpm_host_views *v, uint32_t mask) {
    if (!h || !v) return MPM_E_ARG;
    try {
        if (!h->uploaded) throw Err{MPM_E_STATE, "mpm_download before mpm_upload"};
        CK(cudaSetDevice(h->dev));
        dispatch<Download>(h, v, mask);
        return MPM_OK;
    } catch (const Err &e) { return fail(h, e); }
}

int mpm_snapshot(mpm_handle *h, mpm_h5 *f, int64_t group, double Ti, uint32_t mask, int32_t type) {
    if (!h) return MPM_E_ARG;
    try {
        if (!f) throw Err{MPM_E_ARG, "mpm_snapshot: null file"};
        if (!h->uploaded) throw Err{MPM_E_STATE, "mpm_snapshot before mpm_upload"};
        if (type != MPM_T_F64 && type != MPM_T_F32) throw Err{MPM_E_ARG, "snapshot type must be MPM_T_F64 or MPM_T_F32"};
        const uint32_t allowed = h->ts ? (uint32_t)MPM_F_SNAPSHOT_TS : (uint32_t)MPM_F_SNAPSHOT;
        if (!mask || (mask & ~allowed)) throw Err{MPM_E_ARG, "snapshot fields outside MPM_F_SNAPSHOT(_TS) of this model"};
        if (group < 0) throw Err{MPM_E_ARG, "negative snapshot group"};
        CK(cudaSetDevice(h->dev));
        const int64_t np = h->d.np;
        int64_t ncol = 0;
        for (const SnapField &fd : kSnapFields)
            if (mask & fd.bit) ncol += snap_columns(fd.bit, h->d.dim);
        const size_t bytes = std::max<size_t>(16, (size_t)(ncol * np) * (type == MPM_T_F64 ? 8 : 4));
        SnapState *S = h->snap;
        if (!S) {
            S = new SnapState;
            S->device = h->dev;
            S->np = np;
            S->dim = h->d.dim;
            h->snap = S;
            CK(cudaStreamCreateWithFlags(&S->copy, cudaStreamNonBlocking));
            for (int k = 0; k < 2; ++k) {
                CK(cudaEventCreateWithFlags(&S->gathered[k], cudaEventDisableTiming));
                CK(cudaEventCreateWithFlags(&S->copied[k], cudaEventDisableTiming));
            }
            S->th = std::thread(snap_writer, S);
        }
        std::unique_lock<std::mutex> lk(S->mu);
        if (S->err != MPM_OK) {
            Err e{S->err, S->msg};
            S->err = MPM_OK;
            throw e;
        }
        if (S->cap < bytes) {
            S->cv.wait(lk, [&] { return !S->busy[0] && !S->busy[1]; });
            for (int k = 0; k < 2; ++k) {
                if (S->dev[k]) { cudaFree(S->dev[k]); h->bytes -= S->cap; S->dev[k] = nullptr; }
                if (S->host[k]) { cudaFreeHost(S->host[k]); S->host[k] = nullptr; }
            }
            S->cap = 0;
            for (int k = 0; k < 2; ++k) {
                CK(cudaMalloc(&S->dev[k], bytes));
                h->bytes += bytes;
                CK(cudaMallocHost(&S->host[k], bytes));
            }
            S->cap = bytes;
        }
        const int slot = S->next;
        S->cv.wait(lk, [&] { return !S->busy[slot]; });
        S->busy[slot] = true;
        S->next ^= 1;
        lk.unlock();
        try {
            // gather on the compute stream (after every step issued so far), copy on the copy stream
            dispatch<SnapGather>(h, mask, type, S->dev[slot]);
            CK(cudaEventRecord(S->gathered[slot], h->stream));
            CK(cudaStreamWaitEvent(S->copy, S->gathered[slot], 0));
            CK(cudaMemcpyAsync(S->host[slot], S->dev[slot], bytes, cudaMemcpyDeviceToHost, S->copy));
            CK(cudaEventRecord(S->copied[slot], S->copy));
        } catch (...) {
            std::lock_guard<std::mutex> g(S->mu);
            S->busy[slot] = false;
            throw;
        }
        lk.lock();
        S->q.push_back(SnapJob{slot, f, group, Ti, mask, type});
        S->cv.notify_all();
        return MPM_OK;
    } catch (const Err &e) { return fail(h, e); }
}

int mpm_snapshot_wait(mpm_handle *h, int64_t *written) {
    if (!h) return MPM_E_ARG;
    SnapState *S = h->snap;
    if (!S) {
        if (written) *written = 0;
        return MPM_OK;
    }
    std::unique_lock<std::mutex> lk(S->mu);
    S->cv.wait(lk, [&] { return S->q.empty(); });
    if (written) *written = S->written;
    if (S->err != MPM_OK) {
        const Err e{S->err, S->msg};
        S->err = MPM_OK;
        return fail(h, e);
    }
    return MPM_OK;
}

int mpm_compute_p2c(mpm_handle *h, int64_t *out) {
    if (!h || !out) return MPM_E_ARG;
    try {
        if (!h->uploaded) throw Err{MPM_E_STATE, "mpm_compute_p2c before mpm_upload"};
        CK(cudaSetDevice(h->dev));
        dispatch<P2CAll>(h, out);
        return MPM_OK;
    } catch (const Err &e) { return fail(h, e); }
}

int mpm_download_order(mpm_handle *h, int64_t *out) {
    if (!h || !out) return MPM_E_ARG;
    try {
        CK(cudaSetDevice(h->dev));
        dispatch<Order>(h, out);
        return MPM_OK;
    } catch (const Err &e) { return fail(h, e); }
}

int mpm_sort(mpm_handle *h) {
    if (!h) return MPM_E_ARG;
    try {
        if (!h->uploaded) throw Err{MPM_E_STATE, "mpm_sort before mpm_upload"};
        CK(cudaSetDevice(h->dev));
        dispatch<DoSort>(h);
        CK(cudaStreamSynchronize(h->stream));
        return check_flags(h);
    } catch (const Err &e) { return fail(h, e); }
}

int mpm_run_stages(mpm_handle *h, double dt, double Ti, uint32_t mask) {
    if (!h) return MPM_E_ARG;
    try {
        if (!h->uploaded) throw Err{MPM_E_STATE, "mpm_run_stages before mpm_upload"};
        if (h->ts) throw Err{MPM_E_UNSUPPORTED, "per-stage runs are provided for the one-phase step"};
        CK(cudaSetDevice(h->dev));
        dispatch<Stages>(h, dt, Ti, mask);
        CK(cudaStreamSynchronize(h->stream));
        return check_flags(h);
    } catch (const Err &e) { return fail(h, e); }
}

int mpm_download_grid(mpm_handle *h, int32_t field, double *out) {
    if (!h || !out) return MPM_E_ARG;
    try {
        CK(cudaSetDevice(h->dev));
        CK(cudaStreamSynchronize(h->stream));
        dispatch<GridOut>(h, (int)field, out);
        return MPM_OK;
    } catch (const Err &e) { return fail(h, e); }
}

int mpm_destroy(mpm_handle *h) {
    if (!h) return MPM_OK;
    cudaSetDevice(h->dev);
    if (h->stream) cudaStreamSynchronize(h->stream);
    snap_destroy(h);
    for (void *p : h->allocs) cudaFree(p);
    if (h->graph.exec) cudaGraphExecDestroy(h->graph.exec);
    for (auto e : h->kev) cudaEventDestroy(e);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return MPM_OK;
}

int mpm_get_stats(mpm_handle *h, mpm_stats *s) {
    if (!h || !s) return MPM_E_ARG;
    std::memset(s, 0, sizeof(*s));
    try {
        CK(cudaSetDevice(h->dev));
        if (h->uploaded && h->acc_valid) dispatch<CountActive>(h, &s->active_nodes);
    } catch (const Err &e) { return fail(h, e); }
    s->launches = h->launches;
    s->steps_done = h->steps_done;
    s->sorts_done = h->sorts_done;
    s->error_flags = h->err_host;
    s->kernels_per_step = h->kernels_per_step;
    s->last_step_ms = h->last_step_ms;
    s->device_bytes = (double)h->bytes;
    if (h->surr_stats) {
        unsigned long long st[2] = {0, 0};
        if (cudaMemcpy(st, h->surr_stats, sizeof(st), cudaMemcpyDeviceToHost) == cudaSuccess) {
            s->surr_rows = (int64_t)st[0];
            s->surr_fallbacks = (int64_t)st[1];
        }
    }
    return MPM_OK;
}

const char *mpm_last_error(mpm_handle *h) {
    if (!h) return g_create_error.c_str();
    return h->last_error.c_str();
}

int mpm_abi_sizes(int64_t *desc, int64_t *view, int64_t *views, int64_t *stats) {
    if (desc) *desc = (int64_t)sizeof(mpm_desc);
    if (view) *view = (int64_t)sizeof(mpm_view);
    if (views) *views = (int64_t)sizeof(mpm_host_views);
    if (stats) *stats = (int64_t)sizeof(mpm_stats);
    return MPM_OK;
}

int mpm_set_profiling(mpm_handle *h, int32_t on) {
    if (!h) return MPM_E_ARG;
    h->profiling = on != 0;
    return MPM_OK;
}

int mpm_get_kernel_times(mpm_handle *h, const char **names, double *ms, int64_t *launches, int32_t cap,
                         int32_t *count) {
    if (!h || !count) return MPM_E_ARG;
    int n = (int)std::min<size_t>(h->ktimes.size(), (size_t)std::max(cap, 0));
    for (int i = 0; i < n; ++i) {
        if (names) names[i] = h->ktimes[i].name;
        if (ms) ms[i] = h->ktimes[i].n ? h->ktimes[i].ms / h->ktimes[i].n : 0.0;
        if (launches) launches[i] = h->ktimes[i].n;
    }
    *count = (int32_t)h->ktimes.size();
    return MPM_OK;
}

// Triad A = B + C over growing square FP64 arrays (Tpeak, devicehelpfunc_cuda.jl:102-136).
static __global__ void k_triad(double *A, const double *B, const double *C, int64_t n) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; i < n; i += stride) A[i] = B[i] + C[i];
}

int mpm_peak_bandwidth(int32_t device, double *gbs) {
    if (!gbs) return MPM_E_ARG;
    try {
        CK(cudaSetDevice(device));
        const int64_t n = (int64_t)1 << 27;  // 1 GiB per array
        double *A, *B, *C;
        CK(cudaMalloc(&A, n * 8));
        CK(cudaMalloc(&B, n * 8));
        CK(cudaMalloc(&C, n * 8));
        CK(cudaMemset(B, 0, n * 8));
        CK(cudaMemset(C, 0, n * 8));
        cudaEvent_t e0, e1;
        CK(cudaEventCreate(&e0));
        CK(cudaEventCreate(&e1));
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        float best = 1e30f;
        for (int it = 0; it < 10; ++it) {
            CK(cudaEventRecord(e0));
            k_triad<<<sms * 8, 512>>>(A, B, C, n);
            CK(cudaEventRecord(e1));
            CK(cudaEventSynchronize(e1));
            float ms;
            CK(cudaEventElapsedTime(&ms, e0, e1));
            best = std::min(best, ms);
        }
        *gbs = 3.0 * n * 8 / (best * 1e-3) / 1e9;
        cudaFree(A); cudaFree(B); cudaFree(C);
        cudaEventDestroy(e0); cudaEventDestroy(e1);
        return MPM_OK;
    } catch (const Err &e) {
        g_create_error = e.msg;
        return e.code;
    }
}

}  // extern "C"
