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
    // sources mode
    int ncell;
    const double* state;   // [ns][ncell]
    const double* cc;      // [3][ncell] cell centres
    double* src;           // [4][ncell] m_x, m_y, m_z, E
    double nH_inf, lambda; // cold-model proxy
    int* error;
    // training envelope (sources mode; env_lo null: none): a cell whose
    // features leave [env_lo, env_hi] takes fallback[4][ncell] as its sources
    // (the last Monte-Carlo pass) and is counted in *n_outside
    const float* env_lo;
    const float* env_hi;
    const double* fallback;
    unsigned long long* n_outside;
};

// log of the cold-model neutral density n_inf exp(-lambda theta / (r sin theta)),
// theta the angle from +x, in FP32 (features inside the inference kernel).
__device__ __forceinline__ float log_nh_proxy_f(float n_inf, float lambda, float x, float r) {
    const float c = fminf(fmaxf(x / r, -1.0f), 1.0f);
    const float th = acosf(c);
    const float s = fmaxf(sinf(th), 1e-3f);
    return __logf(n_inf) + fmaxf(-lambda * th / (r * s), -30.0f);
}

// Sources from the network outputs of one cell (sources mode), formed in FP64:
// m_x, m_y, m_z in the frame e1 = V/|V| (radial when V = 0), e2 = the inflow
// direction -x made orthogonal to e1, e3 = e1 x e2; E. For a flow nearly along
// x, e2 = -x - (-x . e1) e1 is a cancellation residue of the transverse
// velocity; in FP32 its direction would be set by rounding noise that the
// flux arithmetic perturbs every step, so the frame is formed in FP64 with the
// same degenerate-case threshold as the training side (closure.py frame()).
__device__ inline void write_sources(const MlpArgs& a, int c, const float* y) {
    const int nc = a.ncell;
    const double rho = a.state[c], vx = a.state[nc + c], vy = a.state[2 * nc + c];
    const double vz = a.state[3 * nc + c];
    const double x = a.cc[c], yy = a.cc[nc + c], z = a.cc[2 * nc + c];
    const double r = sqrt(x * x + yy * yy + z * z);
    const double norm = rho * (double)__expf(log_nh_proxy_f((float)a.nH_inf, (float)a.lambda, (float)x, (float)r));
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
    const double s1 = norm * (double)(y[1] * a.net.oscale[1]), s2 = norm * (double)(y[2] * a.net.oscale[2]);
    const double s3 = norm * (double)(y[3] * a.net.oscale[3]);
    a.src[c] = s1 * e1[0] + s2 * e2[0] + s3 * e3[0];
    a.src[nc + c] = s1 * e1[1] + s2 * e2[1] + s3 * e3[1];
    a.src[2 * nc + c] = s1 * e1[2] + s2 * e2[2] + s3 * e3[2];
    a.src[3 * nc + c] = norm * (double)(y[4] * a.net.oscale[4]);
}

cudaError_t mlp_prepare();  // once per process, before any launch (sets the shared-memory size)
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
