// mpm_grf.cu -- Gaussian random field by the randomised spectral method on the
// device: the evaluation loop of grf_gc! / grf_ec!
// (src/toolkits/randomfield.jl:19-31 compute1!/compute2!, :57-96).
//
//   Y(x) = C · Σ_j ( a_j sin(V_j·x) + b_j cos(V_j·x) )
//
// The harmonics (V_j, a_j, b_j) are drawn on the host (the reference draws
// them with Julia's rand/randn); this entry point only evaluates the sum, one
// thread per point, in FP64 (V·x reaches thousands of radians over a 100 m
// domain, beyond what FP32 argument reduction resolves).
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>

#include "../../include/mpm_b200.h"

namespace mpm_detail {
void set_global_error(const std::string &m);
}

namespace {

constexpr int GRF_CHUNK = 512;   // harmonics staged in shared memory per pass

__global__ void __launch_bounds__(256) k_grf(const double *x, const double *y, const double *z, int64_t np,
                                             const double *harm, int64_t nh, double scale, double *out) {
    __shared__ double sh[GRF_CHUNK * 5];
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const double px = i < np ? x[i] : 0.0, py = i < np ? y[i] : 0.0, pz = (i < np && z) ? z[i] : 0.0;
    double acc = 0.0;
    for (int64_t j0 = 0; j0 < nh; j0 += GRF_CHUNK) {
        const int n = (int)((nh - j0) < GRF_CHUNK ? (nh - j0) : GRF_CHUNK);
        __syncthreads();
        for (int k = threadIdx.x; k < n * 5; k += blockDim.x) sh[k] = harm[j0 * 5 + k];
        __syncthreads();
        for (int j = 0; j < n; ++j) {
            const double *hj = sh + 5 * j;
            const double t = px * hj[0] + py * hj[1] + pz * hj[2];
            double sn, cs;
            sincos(t, &sn, &cs);
            acc += hj[3] * sn + hj[4] * cs;
        }
    }
    if (i < np) out[i] = acc * scale;
}

struct DevBuf {
    void *p = nullptr;
    ~DevBuf() { if (p) cudaFree(p); }
};

}  // namespace

extern "C" int mpm_grf_eval(int32_t device, const double *x, const double *y, const double *z, int64_t np,
                            const double *harm, int64_t nh, double scale, double *out) {
    if (np < 0 || nh < 0 || (np > 0 && (!x || !y || !out)) || (nh > 0 && !harm)) {
        mpm_detail::set_global_error("mpm_grf_eval: invalid arguments");
        return MPM_E_ARG;
    }
    if (np == 0) return MPM_OK;
    auto fail = [](cudaError_t e) {
        mpm_detail::set_global_error(std::string("mpm_grf_eval: ") + cudaGetErrorString(e));
        return MPM_E_CUDA;
    };
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return fail(e);
    DevBuf bx, by, bz, bh, bo;
    const size_t pb = (size_t)np * sizeof(double);
    if ((e = cudaMalloc(&bx.p, pb)) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&by.p, pb)) != cudaSuccess) return fail(e);
    if (z && (e = cudaMalloc(&bz.p, pb)) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&bh.p, (size_t)(nh > 0 ? nh : 1) * 5 * sizeof(double))) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&bo.p, pb)) != cudaSuccess) return fail(e);
    if ((e = cudaMemcpy(bx.p, x, pb, cudaMemcpyHostToDevice)) != cudaSuccess) return fail(e);
    if ((e = cudaMemcpy(by.p, y, pb, cudaMemcpyHostToDevice)) != cudaSuccess) return fail(e);
    if (z && (e = cudaMemcpy(bz.p, z, pb, cudaMemcpyHostToDevice)) != cudaSuccess) return fail(e);
    if (nh > 0 && (e = cudaMemcpy(bh.p, harm, (size_t)nh * 5 * sizeof(double), cudaMemcpyHostToDevice)) != cudaSuccess)
        return fail(e);
    const int64_t blocks = (np + 255) / 256;
    k_grf<<<(unsigned)blocks, 256>>>((const double *)bx.p, (const double *)by.p, (const double *)bz.p, np,
                                     (const double *)bh.p, nh, scale, (double *)bo.p);
    if ((e = cudaGetLastError()) != cudaSuccess) return fail(e);
    if ((e = cudaMemcpy(out, bo.p, pb, cudaMemcpyDeviceToHost)) != cudaSuccess) return fail(e);
    return MPM_OK;
}
