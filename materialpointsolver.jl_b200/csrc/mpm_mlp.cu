// mpm_mlp.cu -- the stress-return surrogate: a 15 -> 64 -> 64 -> 64 -> 6 GELU MLP
// with BF16 weights and FP32 accumulation, run and trained on the sm_100a
// tensor cores (tcgen05.mma, accumulators in TMEM, operands in shared memory).
//
// No counterpart in the reference, whose return mappings (dpP!,
// src/materials/druckerprager.jl:89-155; mcP!, mohrcoulomb.jl) the network
// stands in for.  Features (15, normalised by the caller's mean / std):
// trial stress (6), strain increment (6), accumulated plastic strain, cohesion,
// friction angle.  Output (6): the returned stress, normalised.
//
// Parameters: one FP32 vector (the master copy the optimiser updates), layer
// by layer W[k][n] (k input, n output) then b[n]; the 15-wide input and the
// 6-wide output are padded to 16 with rows / columns that stay zero.  Every
// CTA converts them to BF16 in shared memory in the layouts the MMAs read.
//
// One CTA = 128 threads = one tile of 128 samples (thread t owns sample row t
// and reads TMEM lane t); CTAs stride over the tiles.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>

#include "../../include/mpm_b200.h"
#include "mpm_umma.cuh"

namespace mpm_detail {
void set_global_error(const std::string &m);
}

namespace {

using namespace mpm::umma;

constexpr int TILE = 128;
constexpr int NL = 4;
__host__ __device__ constexpr int lk(int l) { return l == 0 ? 16 : 64; }   // padded inputs of layer l
__host__ __device__ constexpr int ln(int l) { return l == 3 ? 16 : 64; }   // padded outputs of layer l
__host__ __device__ constexpr int ow(int l) {                               // offset of W_l
    return l == 0 ? 0 : l == 1 ? 1088 : l == 2 ? 5248 : 9408;
}
__host__ __device__ constexpr int ob(int l) { return ow(l) + lk(l) * ln(l); }   // offset of b_l
constexpr int NPAR = 10448;
static_assert(ob(3) + 16 == NPAR, "parameter layout");

// norm: in_mean[16], in_std[16], out_mean[16], out_std[16]
constexpr int NORM = 64;

// GELU in the tanh form of Hendrycks & Gimpel (2016), "Gaussian Error Linear
// Units": 0.5 z (1 + tanh(k (z + a z^3))), k = sqrt(2/pi), a = 0.044715, with
// the hardware tanh (tanh.approx.f32).  Its derivative follows from the same
// form: 0.5 (1 + t) + 0.5 z (1 - t^2) k (1 + 3 a z^2), t = tanh(k (z + a z^3)).
__device__ __forceinline__ float tanh_hw(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
constexpr float GELU_K = 0.7978845608028654f, GELU_A = 0.044715f;
__device__ __forceinline__ float gelu(float z) {
    const float t = tanh_hw(GELU_K * z * fmaf(GELU_A * z, z, 1.0f));
    return 0.5f * z * (1.0f + t);
}
__device__ __forceinline__ float gelu_grad(float z) {
    const float t = tanh_hw(GELU_K * z * fmaf(GELU_A * z, z, 1.0f));
    return 0.5f * (1.0f + t) + 0.5f * z * (1.0f - t * t) * GELU_K * fmaf(3.0f * GELU_A * z, z, 1.0f);
}

__device__ __forceinline__ void st_bf16(uint8_t *base, uint32_t off, float v) {
    *reinterpret_cast<__nv_bfloat16 *>(base + off) = __float2bfloat16_rn(v);
}

// 8 consecutive K elements of one row = one 16-byte core-matrix row: one store
__device__ __forceinline__ void st_bf16x8(uint8_t *base, uint32_t off, const float *v) {
    uint4 q;
    __nv_bfloat162 h0 = __floats2bfloat162_rn(v[0], v[1]), h1 = __floats2bfloat162_rn(v[2], v[3]),
                   h2 = __floats2bfloat162_rn(v[4], v[5]), h3 = __floats2bfloat162_rn(v[6], v[7]);
    q.x = *reinterpret_cast<uint32_t *>(&h0);
    q.y = *reinterpret_cast<uint32_t *>(&h1);
    q.z = *reinterpret_cast<uint32_t *>(&h2);
    q.w = *reinterpret_cast<uint32_t *>(&h3);
    *reinterpret_cast<uint4 *>(base + off) = q;
}

// W_l^T (n rows, k columns): B operand of the forward MMA
__device__ void load_wT(uint8_t *dst, const float *P, int l) {
    const int K = lk(l), N = ln(l);
    for (int i = threadIdx.x; i < N * K; i += blockDim.x) {
        const int n = i / K, k = i % K;
        st_bf16(dst, kmajor_offset(n, k, K), P[ow(l) + k * N + n]);
    }
}
// W_l (k rows, n columns): B operand of the backward MMA dY = dZ * W^T
__device__ void load_w(uint8_t *dst, const float *P, int l) {
    const int K = lk(l), N = ln(l);
    for (int i = threadIdx.x; i < N * K; i += blockDim.x) {
        const int k = i / N, n = i % N;
        st_bf16(dst, kmajor_offset(k, n, N), P[ow(l) + k * N + n]);
    }
}

struct Smem {
    uint8_t *wT[NL];      // forward B operands
    uint8_t *x;           // 128 x 16 inputs (A of layer 0)
    uint8_t *a;           // 128 x 64 hidden activations (A of layers 1..3)
    float *bias;          // 4 x 64
    float *norm;          // 64
    uint64_t *bar;
    uint32_t *tslot;
};

__device__ uint8_t *carve(uint8_t *&p, size_t bytes) {
    uint8_t *r = p;
    p += (bytes + 127) & ~(size_t)127;
    return r;
}

__device__ void setup_forward(Smem &S, uint8_t *&p, const float *P, const float *norm) {
    for (int l = 0; l < NL; ++l) S.wT[l] = carve(p, (size_t)lk(l) * ln(l) * 2);
    S.x = carve(p, TILE * 16 * 2);
    S.a = carve(p, TILE * 64 * 2);
    S.bias = reinterpret_cast<float *>(carve(p, 4 * 64 * 4));
    S.norm = reinterpret_cast<float *>(carve(p, NORM * 4));
    S.bar = reinterpret_cast<uint64_t *>(carve(p, 16));
    S.tslot = reinterpret_cast<uint32_t *>(carve(p, 16));
    for (int l = 0; l < NL; ++l) load_wT(S.wT[l], P, l);
    for (int i = threadIdx.x; i < 4 * 64; i += blockDim.x) {
        const int l = i / 64, n = i % 64;
        S.bias[i] = n < ln(l) ? P[ob(l) + n] : 0.0f;
    }
    for (int i = threadIdx.x; i < NORM; i += blockDim.x) S.norm[i] = norm[i];
    fence_proxy_async();   // the weights are read by the tensor core
}

// issue the MMAs of one layer: D[tmem_d] = A (128 x K, at a_saddr) * B^T (N x K)
__device__ __forceinline__ void issue_layer(uint32_t tmem_d, uint32_t a_saddr, uint32_t b_saddr, int K, int N,
                                            uint32_t bar) {
    const uint32_t idesc = idesc_bf16_f32(TILE, N);
    for (int j = 0; j < K / 16; ++j)
        mma_bf16(tmem_d, kstep_desc(a_saddr, j, K), kstep_desc(b_saddr, j, K), idesc, j > 0 ? 1u : 0u);
    commit(bar);
}

// Wait for the MMAs committed to `bar` (phase parity flips per use).  The
// outcome is made CTA-uniform, so a timed-out wait takes every thread out of
// the tile loop together.
__device__ __forceinline__ bool layer_done(uint32_t bar, uint32_t &parity, int *err, int limit = 1 << 20) {
    const bool mine = mbar_wait(bar, parity, limit);
    parity ^= 1u;
    const bool ok = __syncthreads_and(mine) != 0;
    if (!ok && threadIdx.x == 0) atomicOr(err, 1);
    fence_after_sync();
    return ok;
}

// hidden-layer epilogue: bias + GELU of this thread's row -> BF16 row of `a`
__device__ __forceinline__ void hidden_epilogue(uint32_t trow, const float *bias, uint8_t *a, float *zkeep) {
    const int t = threadIdx.x;
#pragma unroll
    for (int c = 0; c < 64; c += 16) {
        float z[16];
        tmem_ld16(trow + c, z);
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            const float zz = z[i] + bias[c + i];
            if (zkeep) zkeep[c + i] = zz;
            z[i] = gelu(zz);
        }
        st_bf16x8(a, kmajor_offset(t, c, 64), z);
        st_bf16x8(a, kmajor_offset(t, c + 8, 64), z + 8);
    }
}

// ---------------------------------------------------------------------------
// Inference: out[i, 0..5] = MLP(feat[i, 0..15]) in physical units.
// flags bit 0: residual (the network predicts out - feat[0..5]); bit 1: the
// timeout test of mpm_mlp_forward (MPM_MLP_TEST_STALL) -- no MMA and no commit
// is issued, so nothing is in flight when the short wait gives up.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(TILE) k_mlp_forward(const float *__restrict__ P, const float *__restrict__ norm,
                                                      const float *__restrict__ feat, float *__restrict__ out,
                                                      int64_t n, const uint32_t *n_dev, int flags, int *err) {
    const int residual = flags & 1;
    const bool stall = (flags & 2) != 0;
    const int limit = stall ? (1 << 10) : (1 << 20);
    if (n_dev) n = min(n, (int64_t)*n_dev);   // rows counted on the device, capped by the buffers
    extern __shared__ __align__(128) uint8_t smem_raw[];
    uint8_t *p = smem_raw;
    Smem S;
    setup_forward(S, p, P, norm);
    const int t = threadIdx.x, w = t >> 5;
    const uint32_t bar = smem_u32(S.bar);
    if (t == 0) mbar_init(bar, 1);
    if (w == 0) tmem_alloc(smem_u32(S.tslot), 64);
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = *S.tslot;
    const uint32_t trow = tmem + ((uint32_t)(w * 32) << 16);
    uint32_t parity = 0;
    bool ok = true;
    const int64_t ntiles = (n + TILE - 1) / TILE;
    for (int64_t tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const int64_t row = tile * TILE + t;
        // inputs: normalise, BF16, canonical layout
        float f[16];
        if (row < n) {
            const float4 *src = reinterpret_cast<const float4 *>(feat + row * 16);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float4 v = src[q];
                f[4 * q] = v.x; f[4 * q + 1] = v.y; f[4 * q + 2] = v.z; f[4 * q + 3] = v.w;
            }
        } else {
#pragma unroll
            for (int k = 0; k < 16; ++k) f[k] = S.norm[k];
        }
        {
            float xn[16];
#pragma unroll
            for (int k = 0; k < 16; ++k) xn[k] = k < 15 ? (f[k] - S.norm[k]) / S.norm[16 + k] : 0.0f;
            st_bf16x8(S.x, kmajor_offset(t, 0, 16), xn);
            st_bf16x8(S.x, kmajor_offset(t, 8, 16), xn + 8);
        }
        fence_proxy_async();
        __syncthreads();
        // layer 0
        if (t == 0 && !stall) {
            fence_after_sync();
            issue_layer(tmem, smem_u32(S.x), smem_u32(S.wT[0]), 16, 64, bar);
        }
        ok = layer_done(bar, parity, err, limit);
        if (!ok) break;
        hidden_epilogue(trow, S.bias, S.a, nullptr);
        fence_before_sync();
        fence_proxy_async();
        __syncthreads();
        // layers 1, 2 (input and output share `a`: the epilogue runs after the MMA completed)
        for (int l = 1; l <= 2 && ok; ++l) {
            if (t == 0) {
                fence_after_sync();
                issue_layer(tmem, smem_u32(S.a), smem_u32(S.wT[l]), 64, 64, bar);
            }
            ok = layer_done(bar, parity, err);
            if (!ok) break;
            hidden_epilogue(trow, S.bias + 64 * l, S.a, nullptr);
            fence_before_sync();
            fence_proxy_async();
            __syncthreads();
        }
        if (!ok) break;
        // layer 3: 16 (6 used) outputs
        if (t == 0) {
            fence_after_sync();
            issue_layer(tmem, smem_u32(S.a), smem_u32(S.wT[3]), 64, 16, bar);
        }
        ok = layer_done(bar, parity, err);
        if (!ok) break;
        float z[16];
        tmem_ld16(trow, z);
        if (row < n) {
#pragma unroll
            for (int o = 0; o < 6; ++o)
                out[row * 6 + o] = (z[o] + S.bias[192 + o]) * S.norm[48 + o] + S.norm[32 + o] + (residual ? f[o] : 0.0f);
        }
        fence_before_sync();
        __syncthreads();
    }
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    if (w == 0) tmem_dealloc(tmem, 64);
}

}  // namespace

namespace mpm_detail {
// 42.5 KB used; 43 KB caps residency at 5 CTAs (320 of 512 TMEM columns) per SM
constexpr size_t MLP_FWD_SMEM = 43 * 1024;
constexpr int MLP_FWD_CTAS_PER_SM = 5;

// Make the forward kernel launchable with its shared memory (call outside any
// stream capture).
__attribute__((visibility("hidden"))) cudaError_t mlp_forward_prepare() {
    return cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MLP_FWD_SMEM);
}

// Forward over min(*n_dev, cap) rows, the count read on the device.
__attribute__((visibility("hidden"))) cudaError_t mlp_forward_dev(const float *P, const float *norm,
                                                                 const float *feat, float *out, int64_t cap,
                                                                 const uint32_t *n_dev, int residual, int *err,
                                                                 cudaStream_t st, int nsm) {
    const int64_t ntiles = (cap + TILE - 1) / TILE;
    const int grid = (int)(ntiles < MLP_FWD_CTAS_PER_SM * nsm ? ntiles : MLP_FWD_CTAS_PER_SM * nsm);
    if (grid < 1) return cudaSuccess;
    k_mlp_forward<<<grid, TILE, MLP_FWD_SMEM, st>>>(P, norm, feat, out, cap, n_dev, residual, err);
    return cudaGetLastError();
}
}  // namespace mpm_detail

extern "C" int mpm_mlp_nparams(void) { return NPAR; }

// Forward pass over n samples; all pointers are DEVICE arrays, work on `stream`.
extern "C" int mpm_mlp_forward(const float *params, const float *norm, const float *feat, float *out, int64_t n,
                               int32_t flags, int *err, void *stream) {
    if (!params || !norm || !err || n < 0 || (n > 0 && (!feat || !out))) {
        mpm_detail::set_global_error("mpm_mlp_forward: invalid arguments");
        return MPM_E_ARG;
    }
    if (n == 0) return MPM_OK;
    const size_t smem = mpm_detail::MLP_FWD_SMEM;
    cudaError_t e = mpm_detail::mlp_forward_prepare();
    if (e == cudaSuccess) {
        int dev = 0, nsm = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        const int64_t ntiles = (n + TILE - 1) / TILE;
        const int grid = (int)(ntiles < mpm_detail::MLP_FWD_CTAS_PER_SM * nsm ? ntiles
                                                                              : mpm_detail::MLP_FWD_CTAS_PER_SM * nsm);
        k_mlp_forward<<<grid, TILE, smem, (cudaStream_t)stream>>>(params, norm, feat, out, n, nullptr, flags & 3, err);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        mpm_detail::set_global_error(std::string("mpm_mlp_forward: ") + cudaGetErrorString(e));
        return MPM_E_CUDA;
    }
    return MPM_OK;
}

namespace {

// ---------------------------------------------------------------------------
// Training: gradient of L = 1/(2 btot) * sum over samples and the 6 outputs of
// (MLP(x) - y)^2 (normalised units), accumulated into grad[NPAR] (FP32,
// reductions from every CTA), and the loss into *loss.
//
// Per tile, forward with the pre-activations kept in TMEM (Z_l at column 64 l),
// then for l = 3 .. 0:
//   dW_l^T = dZ_l^T (128 x 128 samples) * Y_{l-1}            (TMEM column 384)
//   dY_{l-1} = dZ_l (128 samples x N_l) * W_l^T               (TMEM column 256)
//   dZ_{l-1} = dY_{l-1} .* GELU'(Z_{l-1} + b_{l-1})
// Operands: Y_l^T and dZ^T are stored feature-major (samples contiguous) so that
// the sample sum is the MMA's K dimension; rows of dZ^T beyond N_l are not read
// back (row m of D only depends on row m of A).
// ---------------------------------------------------------------------------
// TMEM columns: Z_0..Z_2 at 0/64/128, Z_3 at 192 (16), dY at 224 (64), and one
// dW_l^T accumulator per layer that persists across the CTA's tiles (the
// weight gradient leaves TMEM once per CTA, not once per tile).
constexpr uint32_t COL_DY = 224, TCOLS = 512;
__host__ __device__ constexpr uint32_t col_dw(int l) { return l == 3 ? 288u : l == 2 ? 352u : l == 1 ? 416u : 480u; }
static_assert(col_dw(0) + 16 <= TCOLS, "TMEM budget");

// Sum 16 per-lane values over the warp by recursive halving (16 shuffles):
// returns the full sum of value index *idx; lanes with an odd id hold a copy.
__device__ __forceinline__ float warp_sum16(const float *v, int *idx) {
    const int lane = threadIdx.x & 31;
    float a[8], b[4], c2[2];
    const bool h4 = (lane >> 4) & 1, h3 = (lane >> 3) & 1, h2 = (lane >> 2) & 1, h1 = (lane >> 1) & 1;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const float mine = h4 ? v[8 + i] : v[i], theirs = h4 ? v[i] : v[8 + i];
        a[i] = mine + __shfl_xor_sync(0xffffffffu, theirs, 16);
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const float mine = h3 ? a[4 + i] : a[i], theirs = h3 ? a[i] : a[4 + i];
        b[i] = mine + __shfl_xor_sync(0xffffffffu, theirs, 8);
    }
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        const float mine = h2 ? b[2 + i] : b[i], theirs = h2 ? b[i] : b[2 + i];
        c2[i] = mine + __shfl_xor_sync(0xffffffffu, theirs, 4);
    }
    const float mine = h1 ? c2[1] : c2[0], theirs = h1 ? c2[0] : c2[1];
    float r = mine + __shfl_xor_sync(0xffffffffu, theirs, 2);
    r += __shfl_xor_sync(0xffffffffu, r, 1);
    *idx = (h4 ? 8 : 0) + (h3 ? 4 : 0) + (h2 ? 2 : 0) + (h1 ? 1 : 0);
    return r;
}

// add 16 consecutive per-row values of the CTA's rows into sums[0..15] (smem)
__device__ __forceinline__ void rows_sum16(const float *v, float *sums) {
    int idx;
    const float r = warp_sum16(v, &idx);
    if ((threadIdx.x & 1) == 0 && r != 0.0f) atomicAdd(&sums[idx], r);
}

struct TSmem {
    uint8_t *w[NL];       // W_l (k rows x n), layers 1..3
    uint8_t *xT;          // 16 x 128
    uint8_t *yT[3];       // 64 x 128 each: Y_0..Y_2 feature-major
    uint8_t *dz;          // 128 x N (sample-major)
    uint8_t *dzT;         // 128 x 128 (feature-major, rows >= N unused)
    float *dbias;         // 4 x 64
};

// D (+)= A * B^T over K; `accumulate` decides whether the first K step adds
// to D (later steps always do)
__device__ __forceinline__ void issue_gemm(uint32_t tmem_d, uint32_t a_saddr, uint32_t b_saddr, int K, int N,
                                           bool accumulate = false) {
    const uint32_t idesc = idesc_bf16_f32(TILE, N);
    for (int j = 0; j < K / 16; ++j)
        mma_bf16(tmem_d, kstep_desc(a_saddr, j, K), kstep_desc(b_saddr, j, K), idesc,
                 (j > 0 || accumulate) ? 1u : 0u);
}

__global__ void __launch_bounds__(TILE, 1) k_mlp_grad(const float *__restrict__ P, const float *__restrict__ norm,
                                                      const float *__restrict__ feat,
                                                      const float *__restrict__ target, int64_t n, float inv_btot,
                                                      int residual, float *__restrict__ grad, float *__restrict__ loss,
                                                      int *err) {
    extern __shared__ __align__(128) uint8_t smem_raw[];
    uint8_t *p = smem_raw;
    Smem S;
    setup_forward(S, p, P, norm);
    TSmem T;
    T.w[0] = nullptr;
    for (int l = 1; l < NL; ++l) T.w[l] = carve(p, (size_t)lk(l) * ln(l) * 2);
    T.xT = carve(p, 16 * TILE * 2);
    for (int l = 0; l < 3; ++l) T.yT[l] = carve(p, 64 * TILE * 2);
    T.dz = carve(p, TILE * 64 * 2);
    T.dzT = carve(p, TILE * TILE * 2);
    T.dbias = reinterpret_cast<float *>(carve(p, 4 * 64 * 4));
    for (int l = 1; l < NL; ++l) load_w(T.w[l], P, l);
    for (int i = threadIdx.x; i < TILE * TILE; i += blockDim.x)
        reinterpret_cast<__nv_bfloat16 *>(T.dzT)[i] = __float2bfloat16_rn(0.0f);
    for (int i = threadIdx.x; i < 4 * 64; i += blockDim.x) T.dbias[i] = 0.0f;
    fence_proxy_async();

    const int t = threadIdx.x, w = t >> 5;
    const uint32_t bar = smem_u32(S.bar);
    if (t == 0) mbar_init(bar, 1);
    if (w == 0) tmem_alloc(smem_u32(S.tslot), TCOLS);
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = *S.tslot;
    const uint32_t trow = tmem + ((uint32_t)(w * 32) << 16);
    uint32_t parity = 0;
    bool ok = true;
    float my_loss = 0.0f;
    const int64_t ntiles = (n + TILE - 1) / TILE;
    for (int64_t tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const int64_t row = tile * TILE + t;
        const bool valid = row < n;
        float f[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) f[k] = valid ? feat[row * 16 + k] : S.norm[k];
        {
            float xn[16];
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                xn[k] = k < 15 ? (f[k] - S.norm[k]) / S.norm[16 + k] : 0.0f;
                st_bf16(T.xT, kmajor_offset(k, t, TILE), xn[k]);
            }
            st_bf16x8(S.x, kmajor_offset(t, 0, 16), xn);
            st_bf16x8(S.x, kmajor_offset(t, 8, 16), xn + 8);
        }
        fence_proxy_async();
        __syncthreads();
        // ---- forward, Z_l kept at column 64 l
        for (int l = 0; l < 3 && ok; ++l) {
            if (t == 0) {
                fence_after_sync();
                issue_layer(tmem + 64u * l, smem_u32(l == 0 ? S.x : S.a), smem_u32(S.wT[l]), lk(l), 64, bar);
            }
            ok = layer_done(bar, parity, err);
            if (!ok) break;
#pragma unroll
            for (int c = 0; c < 64; c += 16) {
                float z[16];
                tmem_ld16(trow + 64u * l + c, z);
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    z[i] = gelu(z[i] + S.bias[64 * l + c + i]);
                    st_bf16(T.yT[l], kmajor_offset(c + i, t, TILE), z[i]);
                }
                st_bf16x8(S.a, kmajor_offset(t, c, 64), z);
                st_bf16x8(S.a, kmajor_offset(t, c + 8, 64), z + 8);
            }
            fence_before_sync();
            fence_proxy_async();
            __syncthreads();
        }
        if (!ok) break;
        if (t == 0) {
            fence_after_sync();
            issue_layer(tmem + 192u, smem_u32(S.a), smem_u32(S.wT[3]), 64, 16, bar);
        }
        ok = layer_done(bar, parity, err);
        if (!ok) break;
        // ---- output layer: dZ_3 = (yhat - y) / btot on the 6 outputs
        {
            float z[16];
            tmem_ld16(trow + 192u, z);
#pragma unroll
            for (int o = 0; o < 16; ++o) {
                float d = 0.0f;
                if (valid && o < 6) {
                    const float yh = z[o] + S.bias[192 + o];
                    const float y = (target[row * 6 + o] - (residual ? f[o] : 0.0f) - S.norm[32 + o]) / S.norm[48 + o];
                    d = yh - y;
                    my_loss += 0.5f * d * d * inv_btot;
                    d *= inv_btot;
                }
                st_bf16(T.dzT, kmajor_offset(o, t, TILE), d);
                z[o] = d;
            }
            // the row-major copy as two 16-byte stores (a thread owns its row)
            st_bf16x8(T.dz, kmajor_offset(t, 0, 16), z);
            st_bf16x8(T.dz, kmajor_offset(t, 8, 16), z + 8);
            rows_sum16(z, T.dbias + 192);
        }
        // ---- backward through layers 3, 2, 1 (dW_l and dY_{l-1}), then dW_0
        for (int l = 3; l >= 0 && ok; --l) {
            fence_before_sync();
            fence_proxy_async();
            __syncthreads();
            if (t == 0) {
                fence_after_sync();
                issue_gemm(tmem + col_dw(l), smem_u32(T.dzT), smem_u32(l == 0 ? T.xT : T.yT[l - 1]), TILE, lk(l),
                           tile != (int64_t)blockIdx.x);
                if (l > 0) issue_gemm(tmem + COL_DY, smem_u32(T.dz), smem_u32(T.w[l]), ln(l), lk(l));
                commit(bar);
            }
            ok = layer_done(bar, parity, err);
            if (!ok) break;
            if (l == 0) break;
            // dZ_{l-1} = dY_{l-1} .* GELU'(Z_{l-1} + b_{l-1})
            const int lp = l - 1;
#pragma unroll
            for (int c = 0; c < 64; c += 16) {
                float dy[16], z[16];
                tmem_ld16(trow + COL_DY + c, dy);
                tmem_ld16(trow + 64u * lp + c, z);
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    const float d = valid ? dy[i] * gelu_grad(z[i] + S.bias[64 * lp + c + i]) : 0.0f;
                    st_bf16(T.dzT, kmajor_offset(c + i, t, TILE), d);
                    dy[i] = d;
                }
                st_bf16x8(T.dz, kmajor_offset(t, c, 64), dy);
                st_bf16x8(T.dz, kmajor_offset(t, c + 8, 64), dy + 8);
                rows_sum16(dy, T.dbias + 64 * lp + c);
            }
        }
        fence_before_sync();
        __syncthreads();
    }
    // weight gradients (dW_l^T accumulated over the CTA's tiles: lane = output
    // unit n, columns = inputs k), bias gradients and loss, once per CTA
    __syncthreads();
    fence_after_sync();
    if (ok && (int64_t)blockIdx.x < ntiles) {
        for (int l = 0; l < NL; ++l) {
            const int N = ln(l), K = lk(l);
            for (int c = 0; c < K; c += 16) {
                float g[16];
                tmem_ld16(trow + col_dw(l) + c, g);
                if (t < N) {
#pragma unroll
                    for (int i = 0; i < 16; ++i)
                        if (g[i] != 0.0f) atomicAdd(&grad[ow(l) + (c + i) * N + t], g[i]);
                }
            }
        }
    }
    for (int i = threadIdx.x; i < 4 * 64; i += blockDim.x) {
        const int l = i / 64, nn = i % 64;
        if (nn < ln(l) && T.dbias[i] != 0.0f) atomicAdd(&grad[ob(l) + nn], T.dbias[i]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) my_loss += __shfl_xor_sync(0xffffffffu, my_loss, o);
    if ((t & 31) == 0 && my_loss != 0.0f) atomicAdd(loss, my_loss);
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    if (w == 0) tmem_dealloc(tmem, TCOLS);
}

// Adam on the FP32 master parameters; clears the gradient.
__global__ void k_adam(float *P, float *G, float *M, float *V, int npar, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npar) return;
    const float g = G[i];
    const float m = b1 * M[i] + (1.0f - b1) * g;
    const float v = b2 * V[i] + (1.0f - b2) * g * g;
    M[i] = m;
    V[i] = v;
    P[i] -= lr * (m / c1) / (sqrtf(v / c2) + eps);
    G[i] = 0.0f;
}

}  // namespace

// Gradient of the loss over n samples (feat: n x 16, target: n x 6, DEVICE
// arrays), ADDED to grad[mpm_mlp_nparams()]; the loss is added to *loss.
// inv_btot scales both (1 / batch size for a mean).
extern "C" int mpm_mlp_grad(const float *params, const float *norm, const float *feat, const float *target,
                            int64_t n, float inv_btot, int32_t flags, float *grad, float *loss, int *err,
                            void *stream) {
    if (!params || !norm || !grad || !loss || !err || n < 0 || (n > 0 && (!feat || !target))) {
        mpm_detail::set_global_error("mpm_mlp_grad: invalid arguments");
        return MPM_E_ARG;
    }
    if (n == 0) return MPM_OK;
    const size_t smem = 200 * 1024;   // one CTA per SM: it holds all 512 TMEM columns
    cudaError_t e = cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) {
        int dev = 0, nsm = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        const int64_t ntiles = (n + TILE - 1) / TILE;
        const int grid = (int)(ntiles < nsm ? ntiles : nsm);
        k_mlp_grad<<<grid, TILE, smem, (cudaStream_t)stream>>>(params, norm, feat, target, n, inv_btot, flags & 1,
                                                              grad, loss, err);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        mpm_detail::set_global_error(std::string("mpm_mlp_grad: ") + cudaGetErrorString(e));
        return MPM_E_CUDA;
    }
    return MPM_OK;
}

// One Adam step (bias-corrected with the step count `step` >= 1); zeroes grad.
extern "C" int mpm_mlp_adam(float *params, float *grad, float *m, float *v, float lr, float b1, float b2, float eps,
                            int64_t step, void *stream) {
    if (!params || !grad || !m || !v || step < 1) {
        mpm_detail::set_global_error("mpm_mlp_adam: invalid arguments");
        return MPM_E_ARG;
    }
    const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
    k_adam<<<(NPAR + 255) / 256, 256, 0, (cudaStream_t)stream>>>(params, grad, m, v, NPAR, lr, b1, b2, eps, c1, c2);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        mpm_detail::set_global_error(std::string("mpm_mlp_adam: ") + cudaGetErrorString(e));
        return MPM_E_CUDA;
    }
    return MPM_OK;
}
