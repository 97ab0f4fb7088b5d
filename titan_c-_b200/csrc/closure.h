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
// packed bf16 weights: W1 (128 x 16), W2..W4 (128 x 128), W5 (16 x 128)
constexpr int kWPack = kHid * kInPad + 3 * kHid * kHid + kOutPad * kHid;
constexpr int kBias = 4 * kHid + kOutPad;

struct MlpNet {
    const void* wpack;   // kWPack bf16, canonical K-major blocks (see closure_mlp.cu)
    const float* bias;   // kBias
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
};

__host__ __device__ inline double log_nh_proxy(double n_inf, double lambda, double x, double r) {
    double c = x / r;
    c = c > 1.0 ? 1.0 : (c < -1.0 ? -1.0 : c);
    const double th = acos(c);
    double s = sin(th);
    s = s < 1e-3 ? 1e-3 : s;
    double e = -lambda * th / (r * s);
    e = e < -30.0 ? -30.0 : e;
    return log(n_inf) + e;
}

// Sources from the network outputs of one cell (sources mode).
__device__ inline void write_sources(const MlpArgs& a, int c, const float* y) {
    const int nc = a.ncell;
    const double rho = a.state[c], vx = a.state[nc + c], vy = a.state[2 * nc + c], vz = a.state[3 * nc + c];
    const double x = a.cc[c], yy = a.cc[nc + c], z = a.cc[2 * nc + c];
    const double r = sqrt(x * x + yy * yy + z * z);
    const double norm = rho * exp(log_nh_proxy(a.nH_inf, a.lambda, x, r));
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
    // inflow direction (-x) made orthogonal to e1
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
    const double s1 = norm * y[1] * a.net.oscale[1], s2 = norm * y[2] * a.net.oscale[2];
    const double s3 = norm * y[3] * a.net.oscale[3];
    a.src[c] = s1 * e1[0] + s2 * e2[0] + s3 * e3[0];
    a.src[nc + c] = s1 * e1[1] + s2 * e2[1] + s3 * e3[1];
    a.src[2 * nc + c] = s1 * e1[2] + s2 * e2[2] + s3 * e3[2];
    a.src[3 * nc + c] = norm * y[4] * a.net.oscale[4];
}

cudaError_t mlp_prepare();  // once per process, before any launch (sets the shared-memory size)
cudaError_t launch_mlp_forward(const MlpArgs& a, int mode, int grid, cudaStream_t s);
size_t mlp_forward_smem_bytes();

// A network resident on the device (packed bf16 weights, biases, normalisation).
struct ClosureDev {
    float* params = nullptr;
    void* wpack = nullptr;
    float* bias = nullptr;
    float* norm = nullptr;  // fmean[8], fistd[8], oscale[5]
    int* error = nullptr;
    MlpNet view() const {
        MlpNet n;
        n.wpack = wpack;
        n.bias = bias;
        n.fmean = norm;
        n.fistd = norm + kIn;
        n.oscale = norm + 2 * kIn;
        return n;
    }
};
cudaError_t closure_create(const float* params, const float* norm, ClosureDev* d, cudaStream_t s);
void closure_destroy(ClosureDev* d);

}  // namespace titan
