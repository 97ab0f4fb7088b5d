// Training of the charge-exchange closure on the GPU: BF16 tensor-core GEMMs
// with FP32 accumulation (mma.sync m16n8k16 tiles fed by ldmatrix), the SiLU
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

namespace titan {
namespace train {

constexpr int BM = 64, BN = 64, BK = 32, PAD = 8;

__device__ __forceinline__ void ldmatrix_x4(uint32_t* r, const void* p) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(p);
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(a));
}

__device__ __forceinline__ void ldmatrix_x2(uint32_t* r, const void* p) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(p);
    asm volatile("ldmatrix.sync.aligned.m8n8.x2.shared.b16 {%0,%1}, [%2];" : "=r"(r[0]), "=r"(r[1]) : "r"(a));
}

__device__ __forceinline__ void mma16816(float* c, const uint32_t* a, const uint32_t* b) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// C[M][N] (+)= op(A) op(B); op(A) = A (row-major, lda) or A^T; op(B) = B
// (row-major [K][N], ldb) or B^T (B stored [N][K]). 128 threads, 64x64 tile,
// four warps of 32x32; K split across gridDim.z when `atomic` (C += partial).
template <bool TA, bool TB>
__global__ void __launch_bounds__(128) gemm_kernel(int M, int N, int K, const __nv_bfloat16* __restrict__ A, int lda,
                                                   const __nv_bfloat16* __restrict__ B, int ldb, float* __restrict__ C,
                                                   int ldc, int atomic) {
    __shared__ __align__(16) __nv_bfloat16 As[BM][BK + PAD];
    __shared__ __align__(16) __nv_bfloat16 Bs[BN][BK + PAD];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int kchunks = (K + BK - 1) / BK;
    const int per = (kchunks + gridDim.z - 1) / gridDim.z;
    const int kc0 = blockIdx.z * per, kc1 = min(kchunks, kc0 + per);
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.0f;
    const __nv_bfloat16 zero = __float2bfloat16(0.0f);
    for (int kc = kc0; kc < kc1; ++kc) {
        const int k0 = kc * BK;
        // staging runs along the operand's contiguous dimension in memory, so
        // that a warp's loads coalesce (m for A^T, k for A; n for B, k for B^T)
        for (int i = tid; i < BM * BK; i += 128) {
            const int mm = TA ? i % BM : i / BK, kk = TA ? i / BM : i % BK;
            const int gm = m0 + mm, gk = k0 + kk;
            __nv_bfloat16 v = zero;
            if (gm < M && gk < K) v = TA ? A[(size_t)gk * lda + gm] : A[(size_t)gm * lda + gk];
            As[mm][kk] = v;
        }
        for (int i = tid; i < BN * BK; i += 128) {
            const int nn = TB ? i / BK : i % BN, kk = TB ? i % BK : i / BN;
            const int gn = n0 + nn, gk = k0 + kk;
            __nv_bfloat16 v = zero;
            if (gn < N && gk < K) v = TB ? B[(size_t)gn * ldb + gk] : B[(size_t)gk * ldb + gn];
            Bs[nn][kk] = v;
        }
        __syncthreads();
#pragma unroll
        for (int ks = 0; ks < BK; ks += 16) {
            uint32_t af[2][4], bf[4][2];
#pragma unroll
            for (int i = 0; i < 2; ++i) ldmatrix_x4(af[i], &As[wm + i * 16 + (lane & 15)][ks + 8 * (lane >> 4)]);
#pragma unroll
            for (int j = 0; j < 4; ++j) ldmatrix_x2(bf[j], &Bs[wn + j * 8 + (lane & 7)][ks + 8 * ((lane >> 3) & 1)]);
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) mma16816(acc[i][j], af[i], bf[j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int gm = m0 + wm + i * 16 + (lane >> 2) + (e >= 2 ? 8 : 0);
                const int gn = n0 + wn + j * 8 + 2 * (lane & 3) + (e & 1);
                if (gm < M && gn < N) {
                    float* dst = C + (size_t)gm * ldc + gn;
                    if (atomic)
                        atomicAdd(dst, acc[i][j][e]);
                    else
                        *dst = acc[i][j][e];
                }
            }
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
    dim3 grid((N + train::BN - 1) / train::BN, (M + train::BM - 1) / train::BM, splitk);
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

cudaError_t launch_pack(const float* P, void* out, cudaStream_t s) {
    train::pack_kernel<<<(kWPack + 255) / 256, 256, 0, s>>>(P, static_cast<__nv_bfloat16*>(out));
    return cudaGetLastError();
}

}  // namespace titan
