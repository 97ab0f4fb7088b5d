// tcgen05 building blocks shared by the closure's inference kernel
// (closure_mlp.cu) and its training GEMM (closure_train.cu): the canonical
// K-major shared-memory layout of a BF16 operand, its UMMA descriptor, the
// instruction descriptor of kind::f16 with FP32 accumulation, the MMA and
// commit, tensor-memory loads, the proxy fences, and a bounded sleeping wait
// on an mbarrier.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace titan {
namespace tc {

// ---------------------------------------------------------------------------
// Canonical K-major layout of an R x K bf16 matrix (R rows = M or N, K
// contiguous): core matrix (r/8, k/8) of 8 rows x 8 elements at
// ((k/8) * (R/8) + r/8) * 128 bytes, row r%8 at 16-byte stride.
// ---------------------------------------------------------------------------
__host__ __device__ constexpr int canon_index(int r, int k, int R) {
    return ((k >> 3) * (R >> 3) + (r >> 3)) * 64 + (r & 7) * 8 + (k & 7);
}

// UMMA shared-memory descriptor, SWIZZLE_NONE (layout 0), version 1:
// start >> 4 in [0,14), leading (K-chunk) byte offset >> 4 in [16,30),
// stride (8-row group) byte offset >> 4 in [32,46).
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Instruction descriptor of kind::f16: D f32, A and B bf16, both K-major.
__host__ __device__ constexpr uint32_t instr_desc(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t ad, uint64_t bd, uint32_t idesc, uint32_t accum) {
    const uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
        "l"(ad), "l"(bd), "r"(idesc), "r"(accum), "r"(z), "r"(z), "r"(z), "r"(z));
}

__device__ __forceinline__ void commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Sleeping wait on an mbarrier phase: try_wait with a suspend-time hint of
// 100 us per call, at most ~1 s in total (globaltimer) and 2^14 calls; false
// when it ran out. Waiting threads do not take issue slots from the others.
__device__ __forceinline__ bool mbar_sleep_wait(uint32_t mbar, uint32_t phase) {
    uint64_t t0;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
    for (int it = 0; it < (1 << 14); ++it) {
        uint32_t done = 0;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(phase), "r"(100000u)
            : "memory");
        if (done) return true;
        uint64_t t;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        if (t - t0 > 1000000000ull) return false;
    }
    return false;
}


}  // namespace tc
}  // namespace titan
