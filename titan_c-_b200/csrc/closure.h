// The learned charge-exchange closure: shapes, arguments, and the mapping
// between the network's outputs and the plasma sources.
//
// Inputs (8, standardised with the training set's mean / std):
//   log rho, u_r, |u_t|, log(p/rho), log r, theta (the angle from the upwind
//   axis +x, against which the interstellar medium flows), cos(angle between
//   the plasma velocity and the inflow direction -x), and the log of the
//   cold-model neutral density n_inf exp(-lambda theta / (r sin theta)).
// Outputs (5): the neutral density relative to that proxy, and the plasma
// momentum (3 components in the frame e1 = V/|V|, e2 = the inflow direction
// made orthogonal to e1, e3 = e1 x e2) and energy sources, each divided by
// rho * n_proxy and by the output scale of the training set. The plasma mass
// source of charge exchange is identically zero (Setka_physics.cpp:970), so the
// first output carries the neutral density instead.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "step_types.h"

namespace titan {

constexpr int kIn = 8, kInPad = 16, kHid = 128, kOut = 5, kOutPad = 16, kTile = 128;
constexpr int kModeRaw = 0, kModeSources = 1;
// Packed bf16 operands of the inference kernel, each an N x K block in the
// canonical K-major layout, in this order:
//   W1'  128 x 16: 0.5 W1 for k < 8 and again for 8 <= k < 16 (the input
//        operand carries the features' high BF16 parts at k < 8 and their
//        low parts at k >= 8, so one K = 16 step multiplies both)
//   W2'..W4'  128 x 128: 0.5 W
//   W5   16 x 128
//   B1'..B4'  128 x 16: 0.5 b at k = 0 (multiplied by a constant tile with 1 at k = 0)
//   B5   16 x 16: b5 at k = 0
// The 0.5 makes the hidden-layer accumulator h = (z + b) / 2, so the epilogue
// forms SiLU(z + b) = h (1 + tanh h) without a bias add or a scaling.
// Activations are never rounded to a single BF16: each is carried as a BF16
// pair hi + lo (about 16 significant bits) and every layer multiplies both
// halves by the same weights, which keeps the network a smooth function of
// the cell state (a single BF16 rounding makes it a staircase with steps of
// 2^-8 that turn rounding-level state differences into source jumps).
constexpr int kWPack = kHid * kInPad + 3 * kHid * kHid + kOutPad * kHid + 4 * kHid * kInPad + kOutPad * kInPad;

struct MlpNet {
    const void* wpack;   // kWPack bf16 (above)
    const float* fmean;  // kIn
    const float* fistd;  // kIn
    const float* oscale; // kOut
};

struct MlpArgs {
    MlpNet net;
    int n;                 // rows
    // raw mode
    const float* x;        // [n][kIn] unstandardised features
    float* y;              // [n][kOut]
    // step mode (kModeSources): inputs formed by the previous step's cell
    // update (or closure_inputs), outputs turned into sources by this step's
    int ncell;
    const uint32_t* in_words;  // [8][ncell] standardised inputs as BF16 hi / lo words
    float* y_out;              // [kOut][ncell] network outputs (scaled units)
    int* error;
};

// log of the cold-model neutral density n_inf exp(-lambda theta / (r sin theta)),
// theta the angle from +x, in FP32 (features inside the inference kernel).
__device__ __forceinline__ float log_nh_proxy_f(float n_inf, float lambda, float x, float r) {
    const float c = fminf(fmaxf(x / r, -1.0f), 1.0f);
    const float th = acosf(c);
    const float s = fmaxf(sinf(th), 1e-3f);
    return __logf(n_inf) + fmaxf(-lambda * th / (r * s), -30.0f);
}

// Two FP32 values as BF16 pairs: hi = the nearest BF16 of each (ties away
// from zero), lo = the BF16 nearest the exact remainder v - hi. Returns the
// two packed words {hi(v0), hi(v1)} and {lo(v0), lo(v1)}, element 0 in the
// low half. Integer operations on the bits: adding 2^15 and keeping the top
// 16 bits rounds to nearest; v - hi is exact in FP32.
__device__ __forceinline__ void split_pair(float v0, float v1, uint32_t& hi, uint32_t& lo) {
    const uint32_t r0 = __float_as_uint(v0) + 0x8000u, r1 = __float_as_uint(v1) + 0x8000u;
    const float l0 = v0 - __uint_as_float(r0 & 0xFFFF0000u);
    const float l1 = v1 - __uint_as_float(r1 & 0xFFFF0000u);
    hi = __byte_perm(r0, r1, 0x7632);
    lo = __byte_perm(__float_as_uint(l0) + 0x8000u, __float_as_uint(l1) + 0x8000u, 0x7632);
}

// Input features of one cell (the list above) from its primitives and centre.
// The vector parts are formed in FP64 and rounded once: in FP32 the tangential
// speed sqrt(v^2 - u_r^2) of a nearly radial flow is the square root of a
// cancellation residue (~1e-7 |v|^2, so ~3e-4 |v| of noise with an infinite
// slope), which would make the feature, and the sources, jump with
// rounding-level state changes. |u_t| = |v x r| / r has no cancellation. The
// logarithms take FP32 arguments rounded once from FP64 and use the accurate
// logf, which is continuous at FP32 resolution.
__device__ __forceinline__ void closure_features(double rho, double vx, double vy, double vz, double p, double x,
                                                 double y, double z, double nH_inf, double lambda, float* f) {
    const double r = sqrt(x * x + y * y + z * z);
    const double ir = 1.0 / r;
    const double ur = (vx * x + vy * y + vz * z) * ir;
    const double cx = vy * z - vz * y, cy = vz * x - vx * z, cz = vx * y - vy * x;
    const double ut = sqrt(cx * cx + cy * cy + cz * cz) * ir;
    const double vmag = sqrt(vx * vx + vy * vy + vz * vz);
    f[0] = logf((float)fmax(rho, 1e-30));
    f[1] = (float)ur;
    f[2] = (float)ut;
    f[3] = logf((float)fmax(p / rho, 1e-30));
    f[4] = logf((float)r);
    f[5] = acosf((float)fmin(fmax(x * ir, -1.0), 1.0));
    f[6] = vmag > 0.0 ? (float)(-vx / vmag) : 0.0f;
    f[7] = log_nh_proxy_f((float)nH_inf, (float)lambda, (float)x, (float)r);
}

// The standardised features as the network's input words (hi at K < 8 in
// words 0..3, lo at K >= 8 in words 4..7); whether they leave the envelope.
__device__ __forceinline__ void closure_words(const float* f, const float* norm, const float* env, uint32_t* w8,
                                              bool& outside) {
    outside = false;
    if (env) {
#pragma unroll
        for (int k = 0; k < kIn; ++k) outside |= !(f[k] >= env[k] && f[k] <= env[kIn + k]);
    }
#pragma unroll
    for (int k = 0; k < kIn; k += 2) {
        const float x0 = (f[k] - norm[k]) * norm[kIn + k];
        const float x1 = (f[k + 1] - norm[k + 1]) * norm[kIn + k + 1];
        split_pair(x0, x1, w8[k / 2], w8[kIn / 2 + k / 2]);
    }
}

// Sources m_x, m_y, m_z, E of one cell from the network outputs y (scaled
// units), formed in FP64: momentum in the frame e1 = V/|V| (radial when V = 0),
// e2 = the inflow direction -x made orthogonal to e1, e3 = e1 x e2. For a flow
// nearly along x, e2 = -x - (-x . e1) e1 is a cancellation residue of the
// transverse velocity; in FP32 its direction would be set by rounding noise
// that the flux arithmetic perturbs every step, so the frame is formed in FP64
// with the same degenerate-case threshold as the training side (closure.py
// frame()).
__device__ __forceinline__ void closure_sources(const float* y, const float* oscale, double rho, double vx, double vy,
                                                double vz, double x, double yy, double z, double nH_inf, double lambda,
                                                double* S) {
    const double r = sqrt(x * x + yy * yy + z * z);
    const double norm = rho * (double)__expf(log_nh_proxy_f((float)nH_inf, (float)lambda, (float)x, (float)r));
    const double vm = sqrt(vx * vx + vy * vy + vz * vz);
    double e1[3], e2[3], e3[3];
    if (vm > 0.0) {
        e1[0] = vx / vm;
        e1[1] = vy / vm;
        e1[2] = vz / vm;
    } else {
        e1[0] = x / r;
        e1[1] = yy / r;
        e1[2] = z / r;
    }
    const double d = -e1[0];
    e2[0] = -1.0 - d * e1[0];
    e2[1] = -d * e1[1];
    e2[2] = -d * e1[2];
    double n2 = sqrt(e2[0] * e2[0] + e2[1] * e2[1] + e2[2] * e2[2]);
    if (n2 < 1e-12) {  // flow along x: any perpendicular
        e2[0] = 0.0;
        e2[1] = 1.0;
        e2[2] = 0.0;
        n2 = 1.0;
    }
    e2[0] /= n2;
    e2[1] /= n2;
    e2[2] /= n2;
    e3[0] = e1[1] * e2[2] - e1[2] * e2[1];
    e3[1] = e1[2] * e2[0] - e1[0] * e2[2];
    e3[2] = e1[0] * e2[1] - e1[1] * e2[0];
    const double s1 = norm * (double)(y[1] * oscale[1]), s2 = norm * (double)(y[2] * oscale[2]);
    const double s3 = norm * (double)(y[3] * oscale[3]);
    S[0] = s1 * e1[0] + s2 * e2[0] + s3 * e3[0];
    S[1] = s1 * e1[1] + s2 * e2[1] + s3 * e3[1];
    S[2] = s1 * e1[2] + s2 * e2[2] + s3 * e3[2];
    S[3] = norm * (double)(y[4] * oscale[4]);
}

cudaError_t mlp_prepare();  // once per process, before any launch (sets the shared-memory size)
// The closure's input words and envelope flags of every cell from a state and
// its centres (the first step after the state changed outside the step loop).
cudaError_t launch_closure_inputs(const double* state, const double* cc, int ncell, const float* norm,
                                  const float* env, double nH_inf, double lambda, uint32_t* in, unsigned char* outside,
                                  cudaStream_t s);
// grid: one CTA per SM at most (sm_count), two tiles of 128 rows in flight per CTA
cudaError_t launch_mlp_forward(const MlpArgs& a, int mode, int sm_count, cudaStream_t s);
size_t mlp_forward_smem_bytes();

// A network resident on the device (packed bf16 operands, normalisation).
struct ClosureDev {
    float* params = nullptr;
    void* wpack = nullptr;
    float* norm = nullptr;  // fmean[8], fistd[8], oscale[5]
    int* error = nullptr;
    MlpNet view() const {
        MlpNet n;
        n.wpack = wpack;
        n.fmean = norm;
        n.fistd = norm + kIn;
        n.oscale = norm + 2 * kIn;
        return n;
    }
};
cudaError_t closure_create(const float* params, const float* norm, ClosureDev* d, cudaStream_t s);
void closure_destroy(ClosureDev* d);

// One training step of titan_mlp_train: the batch's first row, the learning
// rate, Adam's bias corrections 1 - beta^t, and the epoch its loss adds to.
struct TrainSched {
    long long r0;
    float lr, c1, c2;
    int epoch;
};

}  // namespace titan
