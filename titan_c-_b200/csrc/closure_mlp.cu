// Learned charge-exchange closure: an MLP 8 -> 128 -> 128 -> 128 -> 128 -> 5
// (SiLU) that maps the local plasma state to the sources the Monte-Carlo
// neutral solver would produce (titan_mc_sources), so the step can run without
// re-tracing neutrals. BF16 weights and activations, FP32 accumulation.
//
// Inference (every step) runs on the 5th-generation tensor cores: one CTA owns
// a tile of 128 cells; the layer weights stay in shared memory for the whole
// kernel in the canonical K-major "interleave" layout (8x16-byte core
// matrices); each layer is M=128 x N x K=16 tcgen05.mma instructions issued by
// one thread with the accumulator in TMEM (128 fp32 columns); the four warps
// read their 32 rows back with tcgen05.ld, apply bias and SiLU, and write the
// next layer's BF16 activations into shared memory. Completion goes through an
// mbarrier whose waits are bounded: a wait that runs out records an error and
// the kernel stops issuing work, releases TMEM and returns.
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

// Bounded wait on an mbarrier phase (non-blocking test_wait polled against the
// global timer: at most ~1 s and 2^26 polls); false when it ran out.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t phase) {
    uint64_t t0;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
    for (int it = 0; it < (1 << 26); ++it) {
        uint32_t done = 0;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(phase)
            : "memory");
        if (done) return true;
        if ((it & 255) == 255) {
            uint64_t t;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
            if (t - t0 > 1000000000ull) return false;
        }
    }
    return false;
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

// SiLU of two values in bf16: z * (1 + tanh(z / 2)) / 2, one packed MUFU op.
__device__ __forceinline__ uint32_t silu_bf16x2(float a, float b) {
    __nv_bfloat162 z = __floats2bfloat162_rn(a, b);
    const __nv_bfloat162 half = __floats2bfloat162_rn(0.5f, 0.5f);
    __nv_bfloat162 h = __hmul2(z, half);
    uint32_t hu = *reinterpret_cast<uint32_t*>(&h), tu;
    asm("tanh.approx.bf16x2 %0, %1;" : "=r"(tu) : "r"(hu));
    __nv_bfloat162 t = *reinterpret_cast<__nv_bfloat162*>(&tu);
    __nv_bfloat162 s = __hfma2(t, half, half);
    __nv_bfloat162 y = __hmul2(z, s);
    return *reinterpret_cast<uint32_t*>(&y);
}

// Shared memory of one CTA (bytes).
struct alignas(128) Smem {
    __nv_bfloat16 w1[kHid * kInPad];    // layer 1, N=128 x K=16
    __nv_bfloat16 w[3][kHid * kHid];    // layers 2..4, N=128 x K=128
    __nv_bfloat16 w5[kOutPad * kHid];   // layer 5, N=16 x K=128
    __nv_bfloat16 x[kTile * kInPad];    // input tile, M=128 x K=16
    __nv_bfloat16 a[kTile * kHid];      // activations, M=128 x K=128
    float bias[4 * kHid + kOutPad];
    float fmean[kIn], fistd[kIn];
    uint64_t mbar;
    uint32_t tmem;
    int abort;
};

// Input features of one cell from its state and centre (see closure.h).
__device__ __forceinline__ void cell_features(const MlpArgs& a, int c, float* f) {
    const int nc = a.ncell;
    const double rho = a.state[c], vx = a.state[nc + c], vy = a.state[2 * nc + c], vz = a.state[3 * nc + c];
    const double p = a.state[4 * nc + c];
    const double x = a.cc[c], y = a.cc[nc + c], z = a.cc[2 * nc + c];
    const double r = sqrt(x * x + y * y + z * z);
    const double ur = (vx * x + vy * y + vz * z) / r;
    const double ut2 = fmax(vx * vx + vy * vy + vz * vz - ur * ur, 0.0);
    const double vmag = sqrt(vx * vx + vy * vy + vz * vz);
    f[0] = (float)log(fmax(rho, 1e-30));
    f[1] = (float)ur;
    f[2] = (float)sqrt(ut2);
    f[3] = (float)log(fmax(p / rho, 1e-30));
    f[4] = (float)log(r);
    f[5] = (float)acos(fmin(fmax(x / r, -1.0), 1.0));
    f[6] = (float)(vmag > 0.0 ? -vx / vmag : 0.0);
    f[7] = (float)log_nh_proxy(a.nH_inf, a.lambda, x, r);
}

template <int MODE>
__global__ void __launch_bounds__(128, 1) mlp_forward_tc(MlpArgs args) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    Smem& S = *reinterpret_cast<Smem*>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5;

    // weights (pre-packed in the canonical layout), biases, normalisation
    {
        const uint4* src = reinterpret_cast<const uint4*>(args.net.wpack);
        uint4* dst = reinterpret_cast<uint4*>(S.w1);
        constexpr int n16 = (kHid * kInPad + 3 * kHid * kHid + kOutPad * kHid) * 2 / 16;
        for (int i = tid; i < n16; i += blockDim.x) dst[i] = src[i];
        for (int i = tid; i < 4 * kHid + kOutPad; i += blockDim.x) S.bias[i] = args.net.bias[i];
        if (tid < kIn) {
            S.fmean[tid] = args.net.fmean[tid];
            S.fistd[tid] = args.net.fistd[tid];
        }
    }
    const uint32_t mbar = smem_u32(&S.mbar);
    if (tid == 0) {
        S.abort = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&S.tmem)),
                     "r"(kHid));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = S.tmem;
    const uint32_t tmem_row = tmem + ((uint32_t)(warp * 32) << 16);  // this warp's 32 lanes
    uint32_t phase = 0;

    const uint32_t idesc_h = instr_desc(kTile, kHid);
    const uint32_t idesc_o = instr_desc(kTile, kOutPad);
    const uint32_t x_base = smem_u32(S.x), a_base = smem_u32(S.a);
    const uint32_t w1_base = smem_u32(S.w1), w5_base = smem_u32(S.w5);
    const int ntiles = (args.n + kTile - 1) / kTile;

    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int row = tile * kTile + tid;
        const bool valid = row < args.n;
        // ---- input features -> x tile (bf16, K padded to 16 with zeros)
        float f[kIn];
        if (MODE == kModeRaw) {
#pragma unroll
            for (int k = 0; k < kIn; ++k) f[k] = valid ? args.x[(size_t)row * kIn + k] : 0.0f;
        } else {
            if (valid)
                cell_features(args, row, f);
            else
#pragma unroll
                for (int k = 0; k < kIn; ++k) f[k] = 0.0f;
        }
        {
            uint32_t packed[kInPad / 2];
#pragma unroll
            for (int k = 0; k < kIn; k += 2) {
                const float f0 = valid ? (f[k] - S.fmean[k]) * S.fistd[k] : 0.0f;
                const float f1 = valid ? (f[k + 1] - S.fmean[k + 1]) * S.fistd[k + 1] : 0.0f;
                __nv_bfloat162 v = __floats2bfloat162_rn(f0, f1);
                packed[k / 2] = *reinterpret_cast<uint32_t*>(&v);
            }
#pragma unroll
            for (int k = kIn; k < kInPad; k += 2) packed[k / 2] = 0u;
            uint4* xr = reinterpret_cast<uint4*>(S.x);
            xr[canon_index(tid, 0, kTile) / 8] = make_uint4(packed[0], packed[1], packed[2], packed[3]);
            xr[canon_index(tid, 8, kTile) / 8] = make_uint4(packed[4], packed[5], packed[6], packed[7]);
        }
        fence_async_smem();
        fence_before();
        __syncthreads();
        fence_after();
        if (S.abort) break;
        // ---- layer 1: D = X (128x16) . W1^T
        if (tid == 0) {
            mma_bf16(tmem, smem_desc(x_base, kTile * 16, 128), smem_desc(w1_base, kHid * 16, 128), idesc_h, 0);
            commit(mbar);
        }
        for (int layer = 0; layer < 4; ++layer) {
            if (!mbar_wait(mbar, phase)) S.abort = 1;
            phase ^= 1;
            fence_after();
            // bias + SiLU -> next activations (this thread's row)
            const float* b = S.bias + layer * kHid;
            uint4* ar = reinterpret_cast<uint4*>(S.a);
#pragma unroll
            for (int c0 = 0; c0 < kHid; c0 += 32) {
                float v[32];
                tmem_ld32(tmem_row + c0, v);
                tmem_wait_ld();
#pragma unroll
                for (int j = 0; j < 32; j += 8) {
                    uint32_t q[4];
#pragma unroll
                    for (int e = 0; e < 4; ++e)
                        q[e] = silu_bf16x2(v[j + 2 * e] + b[c0 + j + 2 * e], v[j + 2 * e + 1] + b[c0 + j + 2 * e + 1]);
                    ar[canon_index(tid, c0 + j, kTile) / 8] = make_uint4(q[0], q[1], q[2], q[3]);
                }
            }
            fence_async_smem();
            fence_before();
            __syncthreads();
            fence_after();
            if (S.abort) break;
            if (tid == 0) {
                if (layer < 3) {
                    const uint32_t wb = smem_u32(S.w[layer]);
#pragma unroll
                    for (int s = 0; s < kHid / 16; ++s)
                        mma_bf16(tmem, smem_desc(a_base + s * 2 * kTile * 16, kTile * 16, 128),
                                 smem_desc(wb + s * 2 * kHid * 16, kHid * 16, 128), idesc_h, s > 0);
                } else {
#pragma unroll
                    for (int s = 0; s < kHid / 16; ++s)
                        mma_bf16(tmem, smem_desc(a_base + s * 2 * kTile * 16, kTile * 16, 128),
                                 smem_desc(w5_base + s * 2 * kOutPad * 16, kOutPad * 16, 128), idesc_o, s > 0);
                }
                commit(mbar);
            }
        }
        if (S.abort) break;
        // ---- output layer
        if (!mbar_wait(mbar, phase)) S.abort = 1;
        phase ^= 1;
        fence_after();
        float y[16];
        tmem_ld16(tmem_row, y);
        tmem_wait_ld();
#pragma unroll
        for (int k = 0; k < kOutPad; ++k) y[k] += S.bias[4 * kHid + k];
        if (valid) {
            if (MODE == kModeRaw) {
#pragma unroll
                for (int k = 0; k < kOut; ++k) args.y[(size_t)row * kOut + k] = y[k];
            } else {
                write_sources(args, row, y);
            }
        }
        fence_before();
        __syncthreads();
        fence_after();
    }
    if (S.abort && tid == 0) atomicExch(args.error, 1);
    fence_before();
    __syncthreads();
    fence_after();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kHid));
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

cudaError_t launch_mlp_forward(const MlpArgs& a, int mode, int grid, cudaStream_t s) {
    const size_t smem = sizeof(mlp::Smem) + 1024;
    if (mode == kModeRaw)
        mlp::mlp_forward_tc<kModeRaw><<<grid, 128, smem, s>>>(a);
    else
        mlp::mlp_forward_tc<kModeSources><<<grid, 128, smem, s>>>(a);
    return cudaGetLastError();
}

size_t mlp_forward_smem_bytes() { return sizeof(mlp::Smem) + 1024; }

}  // namespace titan
