// mpm_umma.cuh -- thin wrappers over the sm_100a tensor-core instructions
// (tcgen05.*) used by the stress-return surrogate (mpm_mlp.cu).
//
// Operands live in shared memory in the canonical K-major, no-swizzle layout
// of the tcgen05 matrix descriptor: 8-row x 16-byte core matrices; inside one
// core matrix the 8 rows are 16 bytes apart; the two 8-element halves of a
// 16-wide K step are LBO = 128 bytes apart; consecutive 8-row groups are
// SBO = (K / 8) * 128 bytes apart.  Element (r, k) of a rows x K bf16 matrix
// sits at byte
//     (r / 8) * K * 16 + (k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2,
// and the operand of the MMA covering K columns [16 j, 16 j + 16) starts at
// byte j * 256 of the matrix.
//
// Accumulators live in tensor memory (TMEM): for M = 128 and cta_group::1,
// row m of D is TMEM lane m and column n is TMEM column (base + n), FP32.
// Warp w of the CTA reads lanes [32 w, 32 w + 32).
//
// Every wait on an mbarrier is bounded: it gives up after a fixed number of
// polls and reports failure, so a fault in the issue sequence cannot hang the
// GPU.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace mpm {
namespace umma {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// byte offset of element (r, k) in the canonical K-major layout with K columns
__host__ __device__ __forceinline__ uint32_t kmajor_offset(int r, int k, int K) {
    return (uint32_t)((r >> 3) * K * 16 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// shared-memory matrix descriptor: SWIZZLE_NONE, version 1 (sm_100)
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;   // descriptor version for sm_100
    return d;                 // base offset 0, legacy LBO mode, layout type 0 (no swizzle)
}

// descriptor of the K-step j of a K-major operand with K columns at saddr
__device__ __forceinline__ uint64_t kstep_desc(uint32_t saddr, int j, int K) {
    return smem_desc(saddr + (uint32_t)j * 256u, 128u, (uint32_t)K * 16u);
}

// instruction descriptor, kind::f16: A = B = BF16, D = F32, both K-major
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D[tmem] (+)= A * B^T over one K = 16 step; issued by one thread
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
        "}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0)
        : "memory");
}

// arrive on the mbarrier once every previously issued MMA of this thread completed
__device__ __forceinline__ void commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void fence_before_sync() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// generic-proxy shared-memory writes -> visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// bounded wait for the given phase parity; false if it never completed
// within `limit` polls
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int limit = 1 << 20) {
    for (int it = 0; it < limit; ++it) {
        uint32_t ok;
        asm volatile(
            "{\n\t"
            ".reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t"
            "}\n"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

// TMEM allocation by one full warp; the base address is written to *slot (smem)
__device__ __forceinline__ void tmem_alloc(uint32_t slot_saddr, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot_saddr), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 16 consecutive FP32 columns of this thread's lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

}  // namespace umma
}  // namespace mpm
