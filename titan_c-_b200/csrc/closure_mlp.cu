// Learned charge-exchange closure: an MLP 8 -> 128 -> 128 -> 128 -> 128 -> 5
// (SiLU) that maps the local plasma state to the sources the Monte-Carlo
// neutral solver would produce (titan_mc_sources), so the step can run without
// re-tracing neutrals. BF16 weights, FP32 accumulation.
//
// Inference (every step) runs on the 5th-generation tensor cores. A CTA holds
// the layer weights in shared memory for the whole kernel, in the canonical
// K-major "interleave" layout (8x16-byte core matrices), and runs two pairs
// of warpgroups, each pair with its own tile of 128 cells in flight. A tile's
// activations live in tensor memory next to its accumulator and are the A
// operand of the next layer's tcgen05.mma (the TMEM-A form), so shared memory
// holds only the weights: while one pair turns its accumulator into the next
// layer's activations (tcgen05.ld, SiLU, tcgen05.st), the tensor core works on
// the other pair's layer. One thread of the pair issues the M=128 x N x K=16
// instructions; completion goes through the pair's mbarrier; waiting threads
// sleep (try_wait with a suspend hint) and the waits are bounded: a wait that
// runs out records an error and the pair stops issuing work; the CTA releases
// TMEM and returns.
//
// Precision: the network must be a smooth function of the cell state. Two
// runs whose states differ at rounding level (the FP64 step and the mixed
// step) must get sources that differ at the same level; a network whose
// activations are rounded once to BF16 is a staircase with 2^-8 steps, and
// its sources jump wherever a state difference crosses a step. So every
// activation and every standardised input is carried as a BF16 pair hi + lo
// (hi = the nearest BF16, lo = the BF16 nearest the exact remainder, together
// about 16 significant bits), each layer multiplies both halves by the same
// BF16 weights (K = 256 per hidden layer: 128 hi columns, then 128 lo
// columns), and SiLU is evaluated in FP32. The hidden-layer operands carry 0.5
// and the biases (closure.h), so the accumulator holds h = (z + b) / 2 and
// SiLU(z + b) = h (1 + tanh h): one tanh.approx.f32 and one FMA per column;
// the hi/lo split is integer arithmetic on the FP32 bits (no conversion
// instructions). Features and sources are formed in FP32.
//
// Training runs the same networks through tcgen05 GEMMs (closure_train.cu).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "closure.h"
#include "tcgen05.cuh"

namespace titan {
namespace mlp {
using namespace tc;

__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// D (TMEM) += A (TMEM, M=128 rows in lanes, 2 bf16 per column along K) . B (shared memory)
__device__ __forceinline__ void mma_bf16_ts(uint32_t tmem_d, uint32_t tmem_a, uint64_t bd, uint32_t idesc,
                                            uint32_t accum) {
    const uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
        "r"(tmem_a), "l"(bd), "r"(idesc), "r"(accum), "r"(z), "r"(z), "r"(z), "r"(z));
}

// 8 consecutive 32-bit columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_st8(uint32_t taddr, const uint32_t* r) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"r"(taddr), "r"(r[0]),
                 "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7])
                 : "memory");
}
__device__ __forceinline__ float tanh_f32(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// SiLU of a pair of columns from the accumulator h = (z + b) / 2 (FP32):
// h (1 + tanh h), split into BF16 hi / lo words.
__device__ __forceinline__ void silu_pair(float h0, float h1, uint32_t& hi, uint32_t& lo) {
    const float a0 = fmaf(h0, tanh_f32(h0), h0);
    const float a1 = fmaf(h1, tanh_f32(h1), h1);
    split_pair(a0, a1, hi, lo);
}

// Two tiles of 128 cells in flight per CTA, each worked by a pair of
// warpgroups: both share the tile's rows (a warp reaches only its lane
// quarter of TMEM, so the two warpgroups take the same 128 lanes) and split
// its 128 accumulator columns, 64 each. One warpgroup of the pair also forms
// the next tile's features while the current tile's last layer runs on the
// tensor core; the other turns the outputs into sources.
constexpr int kPairs = 2;
constexpr int kThreads = 256 * kPairs;
// Registers per thread: 16 warps x 56 take 28,672 of the SM's 65,536, so
// blocks of another kernel (the face flux of the same step: three blocks of
// 128 threads at 96 registers) share the SM with a closure CTA. The epilogue
// works 16 accumulator columns at a time to fit.
constexpr int kMaxRegs = 56;
// TMEM columns of one pair: its FP32 accumulator (128 columns), then its
// activations as the next layer's A operand (128 rows in the lanes, two bf16
// per column along K: columns 0..63 the hi halves of K = 0..127, columns
// 64..127 the lo halves; the input tile uses columns 0..7: hi at K < 8, lo at
// K >= 8).
constexpr uint32_t kColsPerPair = 256, kAccCols = 128, kActLoCols = 64;
constexpr uint32_t kCols = kPairs * kColsPerPair;  // 512: the whole TMEM of the SM
static_assert(kCols <= 512, "tensor memory holds 512 columns");

// Shared memory of one CTA. The operand blocks (w1 .. bw5) are contiguous in
// the order of the packed array (closure.h).
struct alignas(128) Smem {
    __nv_bfloat16 w1[kHid * kInPad];           // W1'  N=128 x K=16 (hi and lo inputs)
    __nv_bfloat16 w[3][kHid * kHid];           // W2'..W4'  N=128 x K=128
    __nv_bfloat16 w5[kOutPad * kHid];          // W5   N=16 x K=128
    __nv_bfloat16 bw[4][kHid * kInPad];        // B1'..B4'  N=128 x K=16
    __nv_bfloat16 bw5[kOutPad * kInPad];       // B5   N=16 x K=16
    __nv_bfloat16 ones[kTile * kInPad];        // M=128 x K=16, 1 at k = 0
    float fmean[kIn], fistd[kIn];
    uint64_t mbar[kPairs];
    uint32_t tmem;
    int abort[kPairs];  // written by the pair's threads before its barrier, read after it
};

// Named barrier of one pair of warpgroups (ids 1..kPairs; 0 is __syncthreads).
__device__ __forceinline__ void pair_sync(int p) {
    asm volatile("bar.sync %0, 256;" ::"r"(p + 1) : "memory");
}

// The input words of one row (hi at K < 8 in words 0..3, lo at K >= 8 in
// words 4..7): standardised and split from raw features, or, in step mode,
// as the previous step's cell update (or closure_inputs) formed them.
template <int MODE>
__device__ __forceinline__ void input_words(const MlpArgs& args, const Smem& S, int cell, uint32_t* w8) {
    const bool valid = cell < args.n;
    if (MODE == kModeRaw) {
#pragma unroll
        for (int k = 0; k < kIn; k += 2) {
            const float x0 = valid ? (args.x[(size_t)cell * kIn + k] - S.fmean[k]) * S.fistd[k] : 0.0f;
            const float x1 = valid ? (args.x[(size_t)cell * kIn + k + 1] - S.fmean[k + 1]) * S.fistd[k + 1] : 0.0f;
            split_pair(x0, x1, w8[k / 2], w8[kIn / 2 + k / 2]);
        }
    } else {
#pragma unroll
        for (int k = 0; k < 8; ++k) w8[k] = valid ? args.in_words[(size_t)k * args.ncell + cell] : 0u;
    }
}

template <int MODE>
__global__ void __maxnreg__(kMaxRegs) mlp_forward_tc(MlpArgs args) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    Smem& S = *reinterpret_cast<Smem*>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5;
    const int wg = tid >> 7;             // warpgroup
    const int p = wg >> 1;               // pair: one tile in flight
    const int h = wg & 1;                // accumulator columns 64 h .. 64 h + 63
    const int row = tid & 127;           // this thread's row of the tile (its TMEM lane)
    const bool leader = h == 0 && row == 0;  // issues the pair's MMAs

    // weights (pre-packed in the canonical layout), the constant tile, normalisation
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
        }
    }
    if (tid == 0) {
        for (int i = 0; i < kPairs; ++i) S.abort[i] = 0;
        for (int i = 0; i < kPairs; ++i)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&S.mbar[i])), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&S.tmem)),
                     "r"(kCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    fence_async_smem();
    fence_before();
    __syncthreads();
    fence_after();
    // this pair's accumulator and activation columns (lane 0), and this
    // warp's lane quarter (a warp reaches lanes 32 (warp % 4) .. + 31)
    const uint32_t acc = S.tmem + (uint32_t)p * kColsPerPair;
    const uint32_t act = acc + kAccCols;
    const uint32_t lane = (uint32_t)((warp & 3) * 32) << 16;
    const uint32_t mbar = smem_u32(&S.mbar[p]);
    uint32_t phase = 0;

    const uint32_t idesc_h = instr_desc(kTile, kHid);
    const uint32_t idesc_o = instr_desc(kTile, kOutPad);
    const uint64_t ones_d = smem_desc(smem_u32(S.ones), kTile * 16, 128);
    const uint32_t w5_base = smem_u32(S.w5);
    const int ntiles = (args.n + kTile - 1) / kTile;
    const int stride = kPairs * gridDim.x;

    // h = 1 loads the next tile's input words during the last hidden layer's
    // MMA, so their latency is off the pair's critical path.
    uint32_t w8[8];
    int tile = blockIdx.x + p * gridDim.x;
    if (h == 1 && tile < ntiles) input_words<MODE>(args, S, tile * kTile + row, w8);
    for (; tile < ntiles; tile += stride) {
        const int cell = tile * kTile + row;
        if (h == 1) {
            tmem_st8(act + lane, w8);
            tmem_wait_st();
        }
        fence_before();
        pair_sync(p);
        fence_after();
        if (S.abort[p]) break;
        // ---- layer 1: H = [X_hi X_lo] (128x16) . W1'^T + 1 . B1'^T
        if (leader) {
            mma_bf16_ts(acc, act, smem_desc(smem_u32(S.w1), kHid * 16, 128), idesc_h, 0);
            mma_bf16(acc, ones_d, smem_desc(smem_u32(S.bw[0]), kHid * 16, 128), idesc_h, 1);
            commit(mbar);
        }
        for (int layer = 0; layer < 4; ++layer) {
            if (!mbar_sleep_wait(mbar, phase)) S.abort[p] = 1;
            phase ^= 1;
            fence_after();
            // h -> SiLU -> this half's columns of the next layer's A operand
            {
                float v[16];
#pragma unroll
                for (int q = 0; q < 4; ++q) {  // 16 columns at a time, so few registers stay live
                    tmem_ld16(acc + lane + 64 * h + 16 * q, v);
                    tmem_wait_ld();
                    uint32_t hi[8], lo[8];
#pragma unroll
                    for (int j = 0; j < 8; ++j) silu_pair(v[2 * j], v[2 * j + 1], hi[j], lo[j]);
                    tmem_st8(act + lane + 32 * h + 8 * q, hi);
                    tmem_st8(act + lane + kActLoCols + 32 * h + 8 * q, lo);
                }
                tmem_wait_st();
            }
            fence_before();
            pair_sync(p);
            fence_after();
            if (S.abort[p]) break;
            if (leader) {
                // K = 256: the hi halves, then the lo halves, against the same weight block
                const bool hidden = layer < 3;
                const uint32_t wb = hidden ? smem_u32(S.w[layer]) : w5_base;
                const uint32_t R = hidden ? kHid : kOutPad;
                const uint32_t idesc = hidden ? idesc_h : idesc_o;
#pragma unroll
                for (int half = 0; half < 2; ++half)
#pragma unroll
                    for (int s = 0; s < kHid / 16; ++s)
                        mma_bf16_ts(acc, act + half * kActLoCols + s * 8,
                                    smem_desc(wb + s * 2 * R * 16, R * 16, 128), idesc, (half | s) != 0);
                const uint32_t bb = hidden ? smem_u32(S.bw[layer + 1]) : smem_u32(S.bw5);
                mma_bf16(acc, ones_d, smem_desc(bb, R * 16, 128), idesc, 1);
                commit(mbar);
            }
            if (layer == 2 && h == 1 && tile + stride < ntiles)
                input_words<MODE>(args, S, (tile + stride) * kTile + row, w8);
        }
        if (S.abort[p]) break;
        // ---- the output layer (N = 16)
        if (!mbar_sleep_wait(mbar, phase)) S.abort[p] = 1;
        phase ^= 1;
        fence_after();
        float y[16];
        if (h == 0) {
            tmem_ld16(acc + lane, y);
            tmem_wait_ld();
        }
        fence_before();
        pair_sync(p);  // the accumulator is free for the next tile
        fence_after();
        if (h == 0 && cell < args.n) {
            if (MODE == kModeRaw) {
#pragma unroll
                for (int k = 0; k < kOut; ++k) args.y[(size_t)cell * kOut + k] = y[k];
            } else {
#pragma unroll
                for (int k = 0; k < kOut; ++k) args.y_out[(size_t)k * args.ncell + cell] = y[k];
            }
        }
    }
    if (S.abort[p] && tid == 256 * p) atomicExch(args.error, 1);
    fence_before();
    __syncthreads();
    fence_after();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(S.tmem), "r"(kCols));
}

}  // namespace mlp

namespace mlp {
// closure_inputs: every cell's input words and envelope flag (closure.h).
__global__ void closure_inputs_kernel(const double* __restrict__ state, const double* __restrict__ cc, int nc,
                                      const float* __restrict__ norm, const float* __restrict__ env, double nH_inf,
                                      double lambda, uint32_t* __restrict__ in, unsigned char* __restrict__ outside) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    float f[kIn];
    closure_features(state[c], state[nc + c], state[2 * nc + c], state[3 * nc + c], state[4 * nc + c], cc[c],
                     cc[nc + c], cc[2 * nc + c], nH_inf, lambda, f);
    uint32_t w8[8];
    bool out = false;
    closure_words(f, norm, env, w8, out);
#pragma unroll
    for (int k = 0; k < 8; ++k) in[(size_t)k * nc + c] = w8[k];
    outside[c] = out ? 1 : 0;
}
}  // namespace mlp

cudaError_t launch_closure_inputs(const double* state, const double* cc, int ncell, const float* norm,
                                  const float* env, double nH_inf, double lambda, uint32_t* in, unsigned char* outside,
                                  cudaStream_t s) {
    mlp::closure_inputs_kernel<<<(ncell + 255) / 256, 256, 0, s>>>(state, cc, ncell, norm, env, nH_inf, lambda, in,
                                                                   outside);
    return cudaGetLastError();
}

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
    const int want = (ntiles + mlp::kPairs - 1) / mlp::kPairs;
    const int grid = want < sm_count ? want : sm_count;
    if (grid <= 0) return cudaSuccess;
    if (mode == kModeRaw)
        mlp::mlp_forward_tc<kModeRaw><<<grid, mlp::kThreads, smem, s>>>(a);
    else
        mlp::mlp_forward_tc<kModeSources><<<grid, mlp::kThreads, smem, s>>>(a);
    return cudaGetLastError();
}

size_t mlp_forward_smem_bytes() { return sizeof(mlp::Smem) + 1024; }

}  // namespace titan
