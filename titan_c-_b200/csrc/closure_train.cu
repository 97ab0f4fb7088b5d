// Training of the charge-exchange closure on the GPU: BF16 GEMMs on the
// 5th-generation tensor cores (tcgen05.mma, FP32 accumulator in tensor
// memory, operands staged in shared memory), the SiLU
// forward/backward, bias gradients, the weighted MSE loss and Adam, all in
// this file's kernels. Layer-wise, for a batch of rows:
//   forward   Z_l = A_{l-1} W_l + b_l, A_l = SiLU(Z_l) (bf16), Y = A_4 W_5 + b_5
//   backward  dY = 2 rw w (Y - T) / n; dW_l = A_{l-1}^T dZ_l; db_l = sum dZ_l;
//             dA_{l-1} = dZ_l W_l^T; dZ_{l-1} = dA_{l-1} SiLU'(Z_{l-1})
// Parameters are FP32 masters [W1 16x128 | b1 | W2 128x128 | b2 | W3 | b3 |
// W4 | b4 | W5 128x16 | b5], W_l stored [in][out] row-major; the GEMMs read
// BF16 copies made after every update.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "closure.h"
#include "tcgen05.cuh"

namespace titan {
namespace train {

using namespace tc;

// Tiles of the training GEMM: 128 rows (the tcgen05 M) by up to 64 columns,
// K staged 32 at a time, two stages in flight.
constexpr int TM = 128, TK = 32, TN = 64;

// Set when a bounded wait of a training GEMM ran out (read by the host API).
__device__ int g_gemm_error;

// Copies the [rows x TK] K-chunk at k0 of op(X) into shared memory in the
// canonical K-major layout (R rows, canon_index), zero outside rows x K.
// op(X)[r][k] = X[r * ld + k] (K contiguous: 16-byte copies of 8 elements),
// or X[k * ld + r] when TR (rows contiguous: element copies, consecutive
// threads along r so the loads coalesce).
template <bool TR>
__device__ __forceinline__ void stage_chunk(__nv_bfloat16* dst, int R, const __nv_bfloat16* __restrict__ X, int ld,
                                            int r0, int rows, int k0, int K) {
    if (!TR) {
        // K and ld are multiples of 8 here (the layer widths), so a 16-byte
        // unit is either wholly inside K or wholly past it
        for (int u = threadIdx.x; u < R * (TK / 8); u += blockDim.x) {
            const int r = u / (TK / 8), k = (u % (TK / 8)) * 8;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (r0 + r < rows && k0 + k < K) v = *reinterpret_cast<const uint4*>(X + (size_t)(r0 + r) * ld + k0 + k);
            *reinterpret_cast<uint4*>(dst + canon_index(r, k, R)) = v;
        }
    } else {
        const __nv_bfloat16 zero = __float2bfloat16(0.0f);
        for (int e = threadIdx.x; e < R * TK; e += blockDim.x) {
            const int r = e % R, k = e / R;
            __nv_bfloat16 v = zero;
            if (r0 + r < rows && k0 + k < K) v = X[(size_t)(k0 + k) * ld + r0 + r];
            dst[canon_index(r, k, R)] = v;
        }
    }
}

// C[M][N] (+)= op(A) op(B) on the tensor cores (tcgen05.mma, kind::f16, FP32
// accumulator in tensor memory). op(A) = A (row-major [M][K], lda) or A^T (A
// stored [K][M]); op(B) = B (row-major [K][N], ldb) or B^T (B stored [N][K]).
// One CTA of 128 threads per tile of 128 rows by 64 columns; K split over
// gridDim.z when `atomic` (C += the slice's partial sum). Each K-chunk
// is staged by all threads into one of two buffers; one thread issues its
// K = 16 steps and commits them to that buffer's mbarrier, which the threads
// wait on before they refill the buffer two chunks later. The epilogue reads
// the accumulator with tcgen05.ld (warp w owns rows 32w .. 32w+31).
template <bool TA, bool TB>
__global__ void __launch_bounds__(128) gemm_kernel(int M, int N, int K, const __nv_bfloat16* __restrict__ A, int lda,
                                                   const __nv_bfloat16* __restrict__ B, int ldb, float* __restrict__ C,
                                                   int ldc, int atomic) {
    __shared__ __align__(128) __nv_bfloat16 As[2][TM * TK];
    __shared__ __align__(128) __nv_bfloat16 Bs[2][TN * TK];
    __shared__ __align__(8) uint64_t mbar[2];
    __shared__ uint32_t tmem_base;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int n0 = blockIdx.x * TN;
    const int NP = (min(TN, N - n0) + 15) & ~15;  // this tile's columns, padded to the MMA's granularity
    const int m0 = blockIdx.y * TM;
    const int kchunks = (K + TK - 1) / TK;
    const int per = (kchunks + gridDim.z - 1) / gridDim.z;
    const int kc0 = blockIdx.z * per, kc1 = min(kchunks, kc0 + per);
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[0])));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[1])));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"(TN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tm = tmem_base;
    const uint32_t idesc = instr_desc(TM, NP);
    bool ok = true;
    int n_chunks = 0;
    for (int kc = kc0; kc < kc1; ++kc, ++n_chunks) {
        const int buf = n_chunks & 1;
        // the MMAs that read this buffer two chunks ago must have finished;
        // the whole block stops if any thread's wait ran out
        const bool w = n_chunks < 2 || mbar_sleep_wait(smem_u32(&mbar[buf]), ((n_chunks >> 1) - 1) & 1);
        if (!__syncthreads_and(w)) {
            ok = false;
            break;
        }
        const int k0 = kc * TK;
        stage_chunk<TA>(As[buf], TM, A, lda, m0, M, k0, K);
        stage_chunk<!TB>(Bs[buf], NP, B, ldb, n0, N, k0, K);
        fence_async_smem();
        fence_before();
        __syncthreads();
        fence_after();
        if (tid == 0) {
            const int ksteps = (min(TK, K - k0) + 15) / 16;
            const uint32_t a0 = smem_u32(As[buf]), b0 = smem_u32(Bs[buf]);
            for (int s = 0; s < ksteps; ++s)
                mma_bf16(tm, smem_desc(a0 + s * 2 * TM * 16, TM * 16, 128), smem_desc(b0 + s * 2 * NP * 16, NP * 16, 128),
                         idesc, (n_chunks > 0 || s > 0) ? 1u : 0u);
            commit(smem_u32(&mbar[buf]));
        }
    }
    // the last commit covers every MMA before it (after a wait that ran out,
    // one more bounded wait, so tensor memory is not freed under running MMAs)
    bool w = true;
    if (n_chunks > 0) {
        const int last = n_chunks - 1;
        w = mbar_sleep_wait(smem_u32(&mbar[last & 1]), (last >> 1) & 1);
        if (!w) mbar_sleep_wait(smem_u32(&mbar[last & 1]), (last >> 1) & 1);
    }
    ok = __syncthreads_and(ok && w) != 0;
    if (!ok && tid == 0) atomicExch(&g_gemm_error, 1);
    fence_after();
    if (ok && n_chunks > 0) {
        const int row = m0 + warp * 32 + lane;
        const uint32_t taddr = tm + ((uint32_t)(warp * 32) << 16);
        for (int c0 = 0; c0 < NP; c0 += 16) {
            float v[16];
            tmem_ld16(taddr + (uint32_t)c0, v);
            tmem_wait_ld();
            if (row < M) {
                float* dst = C + (size_t)row * ldc + n0 + c0;
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    if (n0 + c0 + j >= N) break;
                    if (atomic)
                        atomicAdd(dst + j, v[j]);
                    else
                        dst[j] = v[j];
                }
            }
        }
    }
    fence_before();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tm), "r"(TN));
}

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }
__device__ __forceinline__ float dsilu(float z) {
    const float s = 1.0f / (1.0f + __expf(-z));
    return s * (1.0f + z * (1.0f - s));
}

// Z += bias (in place, FP32); A = bf16(SiLU(Z)) or bf16(Z) when !act.
__global__ void bias_act_kernel(float* Z, const float* b, __nv_bfloat16* A, int rows, int cols, int act) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= (long long)rows * cols) return;
    const int c = (int)(i % cols);
    const float z = Z[i] + b[c];
    Z[i] = z;
    if (A) A[i] = __float2bfloat16(act ? silu(z) : z);
}

// dZ = dA * SiLU'(Z) as bf16.
__global__ void dsilu_kernel(const float* dA, const float* Z, __nv_bfloat16* dZ, long long n) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) dZ[i] = __float2bfloat16(dA[i] * dsilu(Z[i]));
}

// Column sums of a bf16 matrix into db (atomic), for bias gradients; a block
// sums kColsumRows rows, so a batch of a few thousand rows spreads over many SMs.
constexpr int kColsumRows = 32;
__global__ void colsum_kernel(const __nv_bfloat16* X, int rows, int cols, float* db) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    const int r0 = blockIdx.y * kColsumRows, r1 = min(rows, r0 + kColsumRows);
    float s = 0.0f;
    for (int r = r0; r < r1; ++r) s += __bfloat162float(X[(size_t)r * cols + c]);
    atomicAdd(db + c, s);
}

// Weighted MSE on the first kOut columns of Y [rows][16]: loss (atomic) and
// dY = 2 rw_r w_k (Y - T) / rows as bf16 [rows][16] (padding columns 0);
// rw (row weights) may be null (all 1).
__global__ void loss_kernel(const float* Y, const float* T, const float* w, const float* rw, int rows,
                            __nv_bfloat16* dY, float* loss) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.0f;
    if (r < rows) {
        const float wr = rw ? rw[r] : 1.0f;
        for (int k = 0; k < kOutPad; ++k) {
            float g = 0.0f;
            if (k < kOut) {
                const float d = Y[(size_t)r * kOutPad + k] - T[(size_t)r * kOut + k];
                l += wr * w[k] * d * d;
                g = 2.0f * wr * w[k] * d / (float)rows;
            }
            dY[(size_t)r * kOutPad + k] = __float2bfloat16(g);
        }
    }
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, l / (float)rows);
}

// Adam on the FP32 masters; `mask` zeroes the padded input rows of W1 and the
// padded output columns of W5 / b5 so they stay zero.
__global__ void adam_kernel(float* p, const float* g, float* m, float* v, int n, float lr, float b1, float b2,
                            float eps, float c1, float c2, const unsigned char* mask) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (!mask[i]) {
        p[i] = 0.0f;
        return;
    }
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// ---- graph-replayed training: the batch's row offset and Adam scalars come
// from a schedule on the device, indexed by a step counter that the last
// kernel of each batch advances, so one captured batch replays for all.

__global__ void input_sched_kernel(const float* X, const float* mean, const float* istd, __nv_bfloat16* X0, int rows,
                                   const TrainSched* sched, const int* step) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= (long long)rows * kInPad) return;
    const long long r0 = sched[*step].r0;
    const int r = (int)(i / kInPad), k = (int)(i % kInPad);
    X0[i] = __float2bfloat16(k < kIn ? (X[(size_t)(r0 + r) * kIn + k] - mean[k]) * istd[k] : 0.0f);
}

__global__ void loss_sched_kernel(const float* Y, const float* T, const float* w, const float* rw, int rows,
                                  __nv_bfloat16* dY, float* loss_epoch, const TrainSched* sched, const int* step) {
    const TrainSched b = sched[*step];
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.0f;
    if (r < rows) {
        const float wr = rw ? rw[b.r0 + r] : 1.0f;
        for (int k = 0; k < kOutPad; ++k) {
            float g = 0.0f;
            if (k < kOut) {
                const float d = Y[(size_t)r * kOutPad + k] - T[(size_t)(b.r0 + r) * kOut + k];
                l += wr * w[k] * d * d;
                g = 2.0f * wr * w[k] * d / (float)rows;
            }
            dY[(size_t)r * kOutPad + k] = __float2bfloat16(g);
        }
    }
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss_epoch + b.epoch, l / (float)rows);
}

__global__ void adam_sched_kernel(float* p, const float* g, float* m, float* v, int n, float b1, float b2, float eps,
                                  const unsigned char* mask, const TrainSched* sched, const int* step) {
    const TrainSched b = sched[*step];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (!mask[i]) {
        p[i] = 0.0f;
        return;
    }
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= b.lr * (mi / b.c1) / (sqrtf(vi / b.c2) + eps);
}

__global__ void advance_kernel(int* step) { *step += 1; }

__global__ void to_bf16_kernel(const float* x, __nv_bfloat16* y, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = __float2bfloat16(x[i]);
}

// Standardised, bf16, K-padded input rows from raw features.
__global__ void input_kernel(const float* X, const float* mean, const float* istd, __nv_bfloat16* X0, int rows) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= (long long)rows * kInPad) return;
    const int r = (int)(i / kInPad), k = (int)(i % kInPad);
    X0[i] = __float2bfloat16(k < kIn ? (X[(size_t)r * kIn + k] - mean[k]) * istd[k] : 0.0f);
}

// Canonical K-major bf16 pack of the FP32 masters for the tcgen05 kernel
// (the operand list of closure.h): element j of an R x K block is row
// n = (j / 64 % (R / 8)) * 8 + j % 64 / 8, column k = (j / 64 / (R / 8)) * 8 + j % 8.
__global__ void pack_kernel(const float* P, __nv_bfloat16* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kWPack) return;
    // offsets of the layers in the master vector [W1 | b1 | W2 | b2 | ... | W5 | b5]
    const int oW1 = 0, ob1 = kInPad * kHid;
    const int oW2 = ob1 + kHid, ob2 = oW2 + kHid * kHid;
    const int oW3 = ob2 + kHid, ob3 = oW3 + kHid * kHid;
    const int oW4 = ob3 + kHid, ob4 = oW4 + kHid * kHid;
    const int oW5 = ob4 + kHid, ob5 = oW5 + kHid * kOutPad;
    constexpr int sW1 = kHid * kInPad, sW = kHid * kHid, sW5 = kOutPad * kHid, sB = kHid * kInPad;
    int j = i, R, region;
    if (j < sW1) {
        region = 0, R = kHid;
    } else if ((j -= sW1) < 3 * sW) {
        region = 1 + j / sW, R = kHid, j %= sW;
    } else if ((j -= 3 * sW) < sW5) {
        region = 4, R = kOutPad;
    } else if ((j -= sW5) < 4 * sB) {
        region = 5 + j / sB, R = kHid, j %= sB;
    } else {
        j -= 4 * sB;
        region = 9, R = kOutPad;
    }
    const int core = j / 64, within = j % 64;
    const int rgroups = R / 8;
    const int n = (core % rgroups) * 8 + within / 8, k = (core / rgroups) * 8 + within % 8;
    float v = 0.0f;
    switch (region) {
        case 0:  // W1' (K = 16): 0.5 W1 for the features' high parts (k < 8) and low parts (k >= 8)
            v = 0.5f * P[oW1 + (k % kIn) * kHid + n];
            break;
        case 1:
        case 2:
        case 3: {  // W2'..W4'
            const int oW = region == 1 ? oW2 : (region == 2 ? oW3 : oW4);
            v = 0.5f * P[oW + k * kHid + n];
            break;
        }
        case 4:  // W5 (N = 16)
            v = P[oW5 + k * kOutPad + n];
            break;
        case 5:
        case 6:
        case 7:
        case 8: {  // B1'..B4'
            const int ob = region == 5 ? ob1 : (region == 6 ? ob2 : (region == 7 ? ob3 : ob4));
            v = k == 0 ? 0.5f * P[ob + n] : 0.0f;
            break;
        }
        default:  // B5
            v = k == 0 ? P[ob5 + n] : 0.0f;
            break;
    }
    out[i] = __float2bfloat16(v);
}

}  // namespace train

cudaError_t launch_gemm(bool ta, bool tb, int M, int N, int K, const void* A, int lda, const void* B, int ldb,
                        float* C, int ldc, int splitk, cudaStream_t s) {
    // a K-contiguous operand needs K and its leading dimension in multiples of 8
    if ((!ta && (K % 8 || lda % 8)) || (tb && (K % 8 || ldb % 8))) return cudaErrorInvalidValue;
    dim3 grid((N + train::TN - 1) / train::TN, (M + train::TM - 1) / train::TM, splitk);
    const int atomic = splitk > 1 ? 1 : 0;
    auto a = static_cast<const __nv_bfloat16*>(A);
    auto b = static_cast<const __nv_bfloat16*>(B);
    if (!ta && !tb) train::gemm_kernel<false, false><<<grid, 128, 0, s>>>(M, N, K, a, lda, b, ldb, C, ldc, atomic);
    if (!ta && tb) train::gemm_kernel<false, true><<<grid, 128, 0, s>>>(M, N, K, a, lda, b, ldb, C, ldc, atomic);
    if (ta && !tb) train::gemm_kernel<true, false><<<grid, 128, 0, s>>>(M, N, K, a, lda, b, ldb, C, ldc, atomic);
    if (ta && tb) train::gemm_kernel<true, true><<<grid, 128, 0, s>>>(M, N, K, a, lda, b, ldb, C, ldc, atomic);
    return cudaGetLastError();
}

cudaError_t launch_bias_act(float* Z, const float* b, void* A, int rows, int cols, int act, cudaStream_t s) {
    const long long n = (long long)rows * cols;
    train::bias_act_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(Z, b, static_cast<__nv_bfloat16*>(A), rows,
                                                                        cols, act);
    return cudaGetLastError();
}

cudaError_t launch_dsilu(const float* dA, const float* Z, void* dZ, long long n, cudaStream_t s) {
    train::dsilu_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(dA, Z, static_cast<__nv_bfloat16*>(dZ), n);
    return cudaGetLastError();
}

cudaError_t launch_colsum(const void* X, int rows, int cols, float* db, cudaStream_t s) {
    dim3 g((cols + 127) / 128, (rows + train::kColsumRows - 1) / train::kColsumRows);
    train::colsum_kernel<<<g, 128, 0, s>>>(static_cast<const __nv_bfloat16*>(X), rows, cols, db);
    return cudaGetLastError();
}

cudaError_t launch_loss(const float* Y, const float* T, const float* w, const float* rw, int rows, void* dY,
                        float* loss, cudaStream_t s) {
    train::loss_kernel<<<(rows + 255) / 256, 256, 0, s>>>(Y, T, w, rw, rows, static_cast<__nv_bfloat16*>(dY), loss);
    return cudaGetLastError();
}

cudaError_t launch_adam(float* p, const float* g, float* m, float* v, int n, float lr, float b1, float b2, float eps,
                        float c1, float c2, const unsigned char* mask, cudaStream_t s) {
    train::adam_kernel<<<(n + 255) / 256, 256, 0, s>>>(p, g, m, v, n, lr, b1, b2, eps, c1, c2, mask);
    return cudaGetLastError();
}

cudaError_t launch_to_bf16(const float* x, void* y, int n, cudaStream_t s) {
    train::to_bf16_kernel<<<(n + 255) / 256, 256, 0, s>>>(x, static_cast<__nv_bfloat16*>(y), n);
    return cudaGetLastError();
}

cudaError_t launch_input_sched(const float* X, const float* mean, const float* istd, void* X0, int rows,
                               const TrainSched* sched, const int* step, cudaStream_t s) {
    const long long n = (long long)rows * kInPad;
    train::input_sched_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(
        X, mean, istd, static_cast<__nv_bfloat16*>(X0), rows, sched, step);
    return cudaGetLastError();
}

cudaError_t launch_loss_sched(const float* Y, const float* T, const float* w, const float* rw, int rows, void* dY,
                              float* loss_epoch, const TrainSched* sched, const int* step, cudaStream_t s) {
    train::loss_sched_kernel<<<(rows + 255) / 256, 256, 0, s>>>(Y, T, w, rw, rows, static_cast<__nv_bfloat16*>(dY),
                                                                loss_epoch, sched, step);
    return cudaGetLastError();
}

cudaError_t launch_adam_sched(float* p, const float* g, float* m, float* v, int n, float b1, float b2, float eps,
                              const unsigned char* mask, const TrainSched* sched, int* step, cudaStream_t s) {
    train::adam_sched_kernel<<<(n + 255) / 256, 256, 0, s>>>(p, g, m, v, n, b1, b2, eps, mask, sched, step);
    train::advance_kernel<<<1, 1, 0, s>>>(step);
    return cudaGetLastError();
}

cudaError_t launch_input(const float* X, const float* mean, const float* istd, void* X0, int rows, cudaStream_t s) {
    const long long n = (long long)rows * kInPad;
    train::input_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(X, mean, istd, static_cast<__nv_bfloat16*>(X0),
                                                                      rows);
    return cudaGetLastError();
}

// 1 when a training GEMM's bounded wait ran out since the last call (and clears it).
int gemm_error_take() {
    int e = 0;
    cudaMemcpyFromSymbol(&e, train::g_gemm_error, sizeof(int));
    if (e) {
        const int z = 0;
        cudaMemcpyToSymbol(train::g_gemm_error, &z, sizeof(int));
    }
    return e;
}

cudaError_t launch_pack(const float* P, void* out, cudaStream_t s) {
    train::pack_kernel<<<(kWPack + 255) / 256, 256, 0, s>>>(P, static_cast<__nv_bfloat16*>(out));
    return cudaGetLastError();
}

}  // namespace titan
