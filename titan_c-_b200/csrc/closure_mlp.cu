// Learned charge-exchange closure: an MLP 8 -> 128 -> 128 -> 128 -> 128 -> 5
// (SiLU) that maps the local plasma state to the sources the Monte-Carlo
// neutral solver would produce (titan_mc_sources), so the step can run without
// re-tracing neutrals. BF16 weights and activations, FP32 accumulation.
//
// Inference (every step) runs on the 5th-generation tensor cores. A CTA holds
// the layer operands in shared memory for the whole kernel, in the canonical
// K-major "interleave" layout (8x16-byte core matrices), and runs three
// warpgroups, each with its own tile of 128 cells in flight and its own
// 128-column TMEM accumulator: while one warpgroup turns its accumulator into
// the next layer's BF16 activations (tcgen05.ld, SiLU), the tensor core works
// on the other warpgroups' layers. Each layer is M=128 x N x K=16
// tcgen05.mma instructions issued by one thread of the warpgroup; completion
// goes through the warpgroup's mbarrier; waiting threads sleep (try_wait with
// a suspend hint) and the waits are bounded: a wait that runs out records an
// error and the warpgroup stops issuing work; the CTA releases TMEM and
// returns.
//
// The hidden-layer operands carry a factor 0.5 and the biases (closure.h), so
// the accumulator holds h = (z + b) / 2 and the epilogue turns a pair of
// columns into SiLU(z + b) = h (1 + tanh h) with one conversion to bf16x2,
// one tanh.approx.bf16x2 and one bf16x2 FMA. Features and sources are formed
// in FP32 (the network itself is BF16).
//
// Training uses the same networks through mma.sync tiles (closure_train.cu).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "closure.h"

namespace titan {
namespace mlp {

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

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,%"
        "20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
          "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
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

// SiLU of a pair of columns from the accumulator h = (z + b) / 2 (FP32):
// h (1 + tanh h) in bf16x2 — one conversion, one tanh, one FMA.
__device__ __forceinline__ uint32_t silu_pair(float h0, float h1) {
    uint32_t hb, t, y;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(hb) : "f"(h1), "f"(h0));
    asm("tanh.approx.bf16x2 %0, %1;" : "=r"(t) : "r"(hb));
    asm("fma.rn.bf16x2 %0, %1, %2, %1;" : "=r"(y) : "r"(hb), "r"(t));
    return y;
}

constexpr int kGroups = 3;  // warpgroups per CTA, one tile in flight each

// Shared memory of one CTA. The operand blocks (w1 .. bw5) are contiguous in
// the order of the packed array (closure.h).
struct alignas(128) Smem {
    __nv_bfloat16 w1[kHid * kInPad];           // W1'  N=128 x K=16
    __nv_bfloat16 w[3][kHid * kHid];           // W2'..W4'  N=128 x K=128
    __nv_bfloat16 w5[kOutPad * kHid];          // W5   N=16 x K=128
    __nv_bfloat16 bw[3][kHid * kInPad];        // B2'..B4'  N=128 x K=16
    __nv_bfloat16 bw5[kOutPad * kInPad];       // B5   N=16 x K=16
    __nv_bfloat16 ones[kTile * kInPad];        // M=128 x K=16, 1 at k = 0
    __nv_bfloat16 a[kGroups][kTile * kHid];    // activations M=128 x K=128; the input
                                               // tile (K=16) aliases its first 4 KB
    float fmean[kIn], fistd[kIn];
    float env_lo[kIn], env_hi[kIn];
    uint64_t mbar[kGroups];
    uint32_t tmem;
    int abort[kGroups];  // written by the group's own threads before its barrier, read after it
};

// Input features of one cell from its state and centre (closure.h), in FP32.
__device__ __forceinline__ void cell_features(const MlpArgs& a, int c, float* f) {
    const int nc = a.ncell;
    const float rho = (float)a.state[c], vx = (float)a.state[nc + c], vy = (float)a.state[2 * nc + c];
    const float vz = (float)a.state[3 * nc + c], p = (float)a.state[4 * nc + c];
    const float x = (float)a.cc[c], y = (float)a.cc[nc + c], z = (float)a.cc[2 * nc + c];
    const float r = sqrtf(x * x + y * y + z * z);
    const float ir = 1.0f / r;
    const float ur = (vx * x + vy * y + vz * z) * ir;
    const float v2 = vx * vx + vy * vy + vz * vz;
    const float vmag = sqrtf(v2);
    f[0] = __logf(fmaxf(rho, 1e-30f));
    f[1] = ur;
    f[2] = sqrtf(fmaxf(v2 - ur * ur, 0.0f));
    f[3] = __logf(fmaxf(p / rho, 1e-30f));
    f[4] = __logf(r);
    f[5] = acosf(fminf(fmaxf(x * ir, -1.0f), 1.0f));
    f[6] = vmag > 0.0f ? -vx / vmag : 0.0f;
    f[7] = log_nh_proxy_f((float)a.nH_inf, (float)a.lambda, x, r);
}

// Named barrier of one warpgroup (ids 1..kGroups; 0 is __syncthreads).
__device__ __forceinline__ void group_sync(int g) {
    asm volatile("bar.sync %0, 128;" ::"r"(g + 1) : "memory");
}

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

template <int MODE>
__global__ void __launch_bounds__(128 * kGroups, 1) mlp_forward_tc(MlpArgs args) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    Smem& S = *reinterpret_cast<Smem*>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5;
    const int g = tid >> 7;          // warpgroup
    const int row = tid & 127;       // this thread's row of the group's tile
    const bool leader = row == 0;    // issues the group's MMAs

    // operands (pre-packed in the canonical layout), the constant tile, normalisation
    {
        const uint4* src = reinterpret_cast<const uint4*>(args.net.wpack);
        uint4* dst = reinterpret_cast<uint4*>(S.w1);
        constexpr int n16 = kWPack * 2 / 16;
        for (int i = tid; i < n16; i += blockDim.x) dst[i] = src[i];
        uint4* on = reinterpret_cast<uint4*>(S.ones);
        const uint32_t one_lo = 0x3F80u;  // bf16 1.0 in the low half (k = 0)
        for (int r = tid; r < kTile; r += blockDim.x) {
            on[canon_index(r, 0, kTile) / 8] = make_uint4(one_lo, 0u, 0u, 0u);
            on[canon_index(r, 8, kTile) / 8] = make_uint4(0u, 0u, 0u, 0u);
        }
        if (tid < kIn) {
            S.fmean[tid] = args.net.fmean[tid];
            S.fistd[tid] = args.net.fistd[tid];
            S.env_lo[tid] = args.env_lo ? args.env_lo[tid] : -3.0e38f;
            S.env_hi[tid] = args.env_lo ? args.env_hi[tid] : 3.0e38f;
        }
    }
    if (tid == 0) {
        for (int i = 0; i < kGroups; ++i) S.abort[i] = 0;
        for (int i = 0; i < kGroups; ++i)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&S.mbar[i])), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    constexpr uint32_t kCols = kGroups <= 2 ? 256u : 512u;  // power of two >= 128 x groups
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&S.tmem)),
                     "r"(kCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    fence_async_smem();
    fence_before();
    __syncthreads();
    fence_after();
    // this group's accumulator: columns [128 g, 128 g + 128); this warp's 32 lanes
    const uint32_t tmem = S.tmem + (uint32_t)(g * kHid);
    const uint32_t tmem_row = tmem + ((uint32_t)((warp & 3) * 32) << 16);
    const uint32_t mbar = smem_u32(&S.mbar[g]);
    uint32_t phase = 0;

    const uint32_t idesc_h = instr_desc(kTile, kHid);
    const uint32_t idesc_o = instr_desc(kTile, kOutPad);
    const uint32_t a_base = smem_u32(S.a[g]), ones_base = smem_u32(S.ones);
    const uint32_t w1_base = smem_u32(S.w1), w5_base = smem_u32(S.w5), bw5_base = smem_u32(S.bw5);
    const int ntiles = (args.n + kTile - 1) / kTile;
    uint4* ar = reinterpret_cast<uint4*>(S.a[g]);

    for (int tile = blockIdx.x + g * gridDim.x; tile < ntiles; tile += kGroups * gridDim.x) {
        const int cell = tile * kTile + row;
        const bool valid = cell < args.n;
        // ---- input features -> input tile (bf16; k = 8 carries 1 for the bias, 9..15 zero)
        float f[kIn];
        bool outside = false;
        if (MODE == kModeRaw) {
#pragma unroll
            for (int k = 0; k < kIn; ++k) f[k] = valid ? args.x[(size_t)cell * kIn + k] : 0.0f;
        } else {
            if (valid) {
                cell_features(args, cell, f);
#pragma unroll
                for (int k = 0; k < kIn; ++k) outside |= !(f[k] >= S.env_lo[k] && f[k] <= S.env_hi[k]);
            } else {
#pragma unroll
                for (int k = 0; k < kIn; ++k) f[k] = 0.0f;
            }
        }
        {
            uint32_t packed[kIn / 2];
#pragma unroll
            for (int k = 0; k < kIn; k += 2) {
                const float f0 = valid ? (f[k] - S.fmean[k]) * S.fistd[k] : 0.0f;
                const float f1 = valid ? (f[k + 1] - S.fmean[k + 1]) * S.fistd[k + 1] : 0.0f;
                __nv_bfloat162 v = __floats2bfloat162_rn(f0, f1);
                packed[k / 2] = *reinterpret_cast<uint32_t*>(&v);
            }
            ar[canon_index(row, 0, kTile) / 8] = make_uint4(packed[0], packed[1], packed[2], packed[3]);
            ar[canon_index(row, 8, kTile) / 8] = make_uint4(0x3F80u, 0u, 0u, 0u);
        }
        fence_async_smem();
        fence_before();
        group_sync(g);
        fence_after();
        if (S.abort[g]) break;
        // ---- layer 1: H = X' (128x16) . W1'^T  (bias through the 1 at k = 8)
        if (leader) {
            mma_bf16(tmem, smem_desc(a_base, kTile * 16, 128), smem_desc(w1_base, kHid * 16, 128), idesc_h, 0);
            commit(mbar);
        }
        for (int layer = 0; layer < 4; ++layer) {
            if (!mbar_sleep_wait(mbar, phase)) S.abort[g] = 1;
            phase ^= 1;
            fence_after();
            // h -> SiLU -> next activations (this thread's row)
#pragma unroll
            for (int c0 = 0; c0 < kHid; c0 += 32) {
                float v[32];
                tmem_ld32(tmem_row + c0, v);
                tmem_wait_ld();
#pragma unroll
                for (int j = 0; j < 32; j += 8) {
                    uint32_t q[4];
#pragma unroll
                    for (int e = 0; e < 4; ++e) q[e] = silu_pair(v[j + 2 * e], v[j + 2 * e + 1]);
                    ar[canon_index(row, c0 + j, kTile) / 8] = make_uint4(q[0], q[1], q[2], q[3]);
                }
            }
            fence_async_smem();
            fence_before();
            group_sync(g);
            fence_after();
            if (S.abort[g]) break;
            if (leader) {
                if (layer < 3) {
                    const uint32_t wb = smem_u32(S.w[layer]);
#pragma unroll
                    for (int s = 0; s < kHid / 16; ++s)
                        mma_bf16(tmem, smem_desc(a_base + s * 2 * kTile * 16, kTile * 16, 128),
                                 smem_desc(wb + s * 2 * kHid * 16, kHid * 16, 128), idesc_h, s > 0);
                    mma_bf16(tmem, smem_desc(ones_base, kTile * 16, 128),
                             smem_desc(smem_u32(S.bw[layer]), kHid * 16, 128), idesc_h, 1);
                } else {
#pragma unroll
                    for (int s = 0; s < kHid / 16; ++s)
                        mma_bf16(tmem, smem_desc(a_base + s * 2 * kTile * 16, kTile * 16, 128),
                                 smem_desc(w5_base + s * 2 * kOutPad * 16, kOutPad * 16, 128), idesc_o, s > 0);
                    mma_bf16(tmem, smem_desc(ones_base, kTile * 16, 128), smem_desc(bw5_base, kOutPad * 16, 128),
                             idesc_o, 1);
                }
                commit(mbar);
            }
        }
        if (S.abort[g]) break;
        // ---- output layer (bias included)
        if (!mbar_sleep_wait(mbar, phase)) S.abort[g] = 1;
        phase ^= 1;
        fence_after();
        float y[16];
        tmem_ld16(tmem_row, y);
        tmem_wait_ld();
        if (valid) {
            if (MODE == kModeRaw) {
#pragma unroll
                for (int k = 0; k < kOut; ++k) args.y[(size_t)cell * kOut + k] = y[k];
            } else if (outside && args.fallback) {
                // outside the training envelope: the last Monte-Carlo sources
#pragma unroll
                for (int k = 0; k < 4; ++k) args.src[k * args.ncell + cell] = args.fallback[k * args.ncell + cell];
            } else {
                write_sources(args, cell, y);
            }
        }
        if (MODE == kModeSources && args.n_outside) {
            const unsigned int bal = __ballot_sync(0xffffffffu, valid && outside);
            if ((threadIdx.x & 31) == 0 && bal) atomicAdd(args.n_outside, (unsigned long long)__popc(bal));
        }
        fence_before();
        group_sync(g);
        fence_after();
    }
    if (S.abort[g] && row == 0) atomicExch(args.error, 1);
    fence_before();
    __syncthreads();
    fence_after();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(S.tmem), "r"(kCols));
}

}  // namespace mlp

cudaError_t mlp_prepare() {
    const int smem = (int)(sizeof(mlp::Smem) + 1024);
    cudaError_t e =
        cudaFuncSetAttribute(mlp::mlp_forward_tc<kModeRaw>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (!e)
        e = cudaFuncSetAttribute(mlp::mlp_forward_tc<kModeSources>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    return e;
}

cudaError_t launch_mlp_forward(const MlpArgs& a, int mode, int sm_count, cudaStream_t s) {
    const size_t smem = sizeof(mlp::Smem) + 1024;
    const int ntiles = (a.n + kTile - 1) / kTile;
    const int want = (ntiles + mlp::kGroups - 1) / mlp::kGroups;
    const int grid = want < sm_count ? want : sm_count;
    if (grid <= 0) return cudaSuccess;
    if (mode == kModeRaw)
        mlp::mlp_forward_tc<kModeRaw><<<grid, 128 * mlp::kGroups, smem, s>>>(a);
    else
        mlp::mlp_forward_tc<kModeSources><<<grid, 128 * mlp::kGroups, smem, s>>>(a);
    return cudaGetLastError();
}

size_t mlp_forward_smem_bytes() { return sizeof(mlp::Smem) + 1024; }

}  // namespace titan
