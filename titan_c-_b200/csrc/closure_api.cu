// Host side of the closure: inference on host buffers, GPU training, and the
// gradient of one batch (for the CPU gradient check).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/titan_b200.h"
#include "closure.h"

namespace titan {
void set_last_error(const std::string& msg);

cudaError_t launch_gemm(bool ta, bool tb, int M, int N, int K, const void* A, int lda, const void* B, int ldb,
                        float* C, int ldc, int splitk, cudaStream_t s);
cudaError_t launch_bias_act(float* Z, const float* b, void* A, int rows, int cols, int act, cudaStream_t s);
cudaError_t launch_dsilu(const float* dA, const float* Z, void* dZ, long long n, cudaStream_t s);
cudaError_t launch_colsum(const void* X, int rows, int cols, float* db, cudaStream_t s);
cudaError_t launch_loss(const float* Y, const float* T, const float* w, const float* rw, int rows, void* dY,
                        float* loss, cudaStream_t s);
cudaError_t launch_adam(float* p, const float* g, float* m, float* v, int n, float lr, float b1, float b2, float eps,
                        float c1, float c2, const unsigned char* mask, cudaStream_t s);
cudaError_t launch_to_bf16(const float* x, void* y, int n, cudaStream_t s);
cudaError_t launch_input(const float* X, const float* mean, const float* istd, void* X0, int rows, cudaStream_t s);
cudaError_t launch_input_sched(const float* X, const float* mean, const float* istd, void* X0, int rows,
                               const TrainSched* sched, const int* step, cudaStream_t s);
cudaError_t launch_loss_sched(const float* Y, const float* T, const float* w, const float* rw, int rows, void* dY,
                              float* loss_epoch, const TrainSched* sched, const int* step, cudaStream_t s);
cudaError_t launch_adam_sched(float* p, const float* g, float* m, float* v, int n, float b1, float b2, float eps,
                              const unsigned char* mask, const TrainSched* sched, int* step, cudaStream_t s);
cudaError_t launch_pack(const float* P, void* out, cudaStream_t s);
int gemm_error_take();

namespace {

// offsets of the layers in the FP32 master vector
constexpr int oW1 = 0, ob1 = kInPad * kHid, oW2 = ob1 + kHid, ob2 = oW2 + kHid * kHid, oW3 = ob2 + kHid,
              ob3 = oW3 + kHid * kHid, oW4 = ob3 + kHid, ob4 = oW4 + kHid * kHid, oW5 = ob4 + kHid,
              ob5 = oW5 + kHid * kOutPad, kNParam = ob5 + kOutPad;
static_assert(kNParam == TITAN_MLP_NPARAM, "parameter count");

int mfail(int code, const std::string& m) {
    set_last_error(m);
    return code;
}

struct Buf {
    std::vector<void*> ptrs;
    cudaError_t err = cudaSuccess;
    template <typename T>
    T* get(size_t n) {
        void* p = nullptr;
        if (err == cudaSuccess && n) err = cudaMalloc(&p, n * sizeof(T));
        ptrs.push_back(p);
        return static_cast<T*>(p);
    }
    ~Buf() {
        for (void* p : ptrs)
            if (p) cudaFree(p);
    }
};

// Device copies of a network: FP32 masters, packed bf16 operands, normalisation.
struct DevNet {
    float* params;
    void* wpack;
    float* norm;  // fmean[8], fistd[8], oscale[5]
    MlpNet view() const {
        MlpNet n;
        n.wpack = wpack;
        n.fmean = norm;
        n.fistd = norm + kIn;
        n.oscale = norm + 2 * kIn;
        return n;
    }
};

cudaError_t upload_net(Buf& b, const float* params, const float* norm, DevNet& d, cudaStream_t s) {
    d.params = b.get<float>(kNParam);
    d.wpack = b.get<uint16_t>(kWPack);
    d.norm = b.get<float>(2 * kIn + kOut);
    if (b.err) return b.err;
    cudaError_t e = cudaMemcpyAsync(d.params, params, sizeof(float) * kNParam, cudaMemcpyHostToDevice, s);
    if (!e) e = cudaMemcpyAsync(d.norm, norm, sizeof(float) * (2 * kIn + kOut), cudaMemcpyHostToDevice, s);
    if (!e) e = launch_pack(d.params, d.wpack, s);
    return e;
}

// Buffers of one training batch and the forward / backward passes on them.
struct Trainer {
    int rows;
    __nv_bfloat16_raw* X0;  // [rows][16] bf16 (stored as raw halves)
    float* Z[5];            // pre-activations [rows][128] (Z[4]: outputs [rows][16])
    void* A[4];             // bf16 activations [rows][128]
    void* Wb;               // bf16 copy of the masters
    float* dA;              // [rows][128]
    void* dZ;               // bf16 [rows][128]
    void* dY;               // bf16 [rows][16]
    float* grad;            // [kNParam]
    float* loss;
};

const int kLayIn[5] = {kInPad, kHid, kHid, kHid, kHid};
const int kLayOut[5] = {kHid, kHid, kHid, kHid, kOutPad};
const int kLayW[5] = {oW1, oW2, oW3, oW4, oW5};
const int kLayB[5] = {ob1, ob2, ob3, ob4, ob5};

cudaError_t forward(Trainer& t, const float* params, cudaStream_t s) {
    cudaError_t e = launch_to_bf16(params, t.Wb, kNParam, s);
    const char* Wb = static_cast<const char*>(t.Wb);
    const void* in = t.X0;
    for (int l = 0; l < 5 && !e; ++l) {
        e = launch_gemm(false, false, t.rows, kLayOut[l], kLayIn[l], in, kLayIn[l], Wb + 2 * (size_t)kLayW[l],
                        kLayOut[l], t.Z[l], kLayOut[l], 1, s);
        if (!e) e = launch_bias_act(t.Z[l], params + kLayB[l], l < 4 ? t.A[l] : nullptr, t.rows, kLayOut[l], 1, s);
        if (l < 4) in = t.A[l];
    }
    return e;
}

// Gradients of one batch: `loss` forms dY (and adds up the loss); then the
// layers backwards.
template <typename Loss>
cudaError_t backward_with(Trainer& t, Loss loss, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(t.grad, 0, sizeof(float) * kNParam, s);
    if (!e) e = loss();
    const char* Wb = static_cast<const char*>(t.Wb);
    const void* dZl = t.dY;
    // dW = A^T dZ has K = the batch's rows: split it so a batch of a few
    // thousand rows still spreads over tens of CTAs (two 32-row chunks or more each)
    const int split = std::max(1, std::min(64, t.rows / 64));
    for (int l = 4; l >= 0 && !e; --l) {
        const void* Ain = l > 0 ? t.A[l - 1] : (const void*)t.X0;
        // dW_l = A_{l-1}^T dZ_l  ([in][out]), db_l = colsum dZ_l
        e = launch_gemm(true, false, kLayIn[l], kLayOut[l], t.rows, Ain, kLayIn[l], dZl, kLayOut[l],
                        t.grad + kLayW[l], kLayOut[l], split, s);
        if (!e) e = launch_colsum(dZl, t.rows, kLayOut[l], t.grad + kLayB[l], s);
        if (l > 0 && !e) {
            // dA_{l-1} = dZ_l W_l^T; dZ_{l-1} = dA SiLU'(Z_{l-1})
            e = launch_gemm(false, true, t.rows, kLayIn[l], kLayOut[l], dZl, kLayOut[l], Wb + 2 * (size_t)kLayW[l],
                            kLayOut[l], t.dA, kLayIn[l], 1, s);
            if (!e) e = launch_dsilu(t.dA, t.Z[l - 1], t.dZ, (long long)t.rows * kHid, s);
            dZl = t.dZ;
        }
    }
    return e;
}

cudaError_t backward(Trainer& t, const float* T, const float* w, const float* rw, cudaStream_t s) {
    return backward_with(t, [&] {
        cudaError_t e = cudaMemsetAsync(t.loss, 0, sizeof(float), s);
        return e ? e : launch_loss(t.Z[4], T, w, rw, t.rows, t.dY, t.loss, s);
    }, s);
}

bool alloc_trainer(Buf& b, Trainer& t, int rows) {
    t.rows = rows;
    t.X0 = b.get<__nv_bfloat16_raw>((size_t)rows * kInPad);
    for (int l = 0; l < 5; ++l) t.Z[l] = b.get<float>((size_t)rows * kLayOut[l]);
    for (int l = 0; l < 4; ++l) t.A[l] = b.get<uint16_t>((size_t)rows * kHid);
    t.Wb = b.get<uint16_t>(kNParam);
    t.dA = b.get<float>((size_t)rows * kHid);
    t.dZ = b.get<uint16_t>((size_t)rows * kHid);
    t.dY = b.get<uint16_t>((size_t)rows * kOutPad);
    t.grad = b.get<float>(kNParam);
    t.loss = b.get<float>(1);
    return b.err == cudaSuccess;
}

std::vector<unsigned char> param_mask() {
    std::vector<unsigned char> m(kNParam, 1);
    for (int i = kIn; i < kInPad; ++i)
        for (int j = 0; j < kHid; ++j) m[oW1 + i * kHid + j] = 0;  // padded input rows
    for (int i = 0; i < kHid; ++i)
        for (int j = kOut; j < kOutPad; ++j) m[oW5 + i * kOutPad + j] = 0;  // padded outputs
    for (int j = kOut; j < kOutPad; ++j) m[ob5 + j] = 0;
    return m;
}

}  // namespace

cudaError_t closure_create(const float* params, const float* norm, ClosureDev* d, cudaStream_t s) {
    cudaError_t e = mlp_prepare();
    if (!e) e = cudaMalloc((void**)&d->params, sizeof(float) * kNParam);
    if (!e) e = cudaMalloc(&d->wpack, sizeof(uint16_t) * kWPack);
    if (!e) e = cudaMalloc((void**)&d->norm, sizeof(float) * (2 * kIn + kOut));
    if (!e) e = cudaMalloc((void**)&d->error, sizeof(int));
    if (!e) e = cudaMemcpyAsync(d->params, params, sizeof(float) * kNParam, cudaMemcpyHostToDevice, s);
    if (!e) e = cudaMemcpyAsync(d->norm, norm, sizeof(float) * (2 * kIn + kOut), cudaMemcpyHostToDevice, s);
    if (!e) e = cudaMemsetAsync(d->error, 0, sizeof(int), s);
    if (!e) e = launch_pack(d->params, d->wpack, s);
    if (!e) e = cudaStreamSynchronize(s);
    return e;
}

void closure_destroy(ClosureDev* d) {
    void* ps[] = {d->params, d->wpack, d->norm, d->error};
    for (void* p : ps)
        if (p) cudaFree(p);
    *d = ClosureDev{};
}

}  // namespace titan

using namespace titan;

extern "C" {

int titan_mlp_forward(const float* params, const float* norm, const float* X, int64_t n, float* Y) {
    if (!params || !norm || !X || !Y || n <= 0) return mfail(TITAN_EINVAL, "titan_mlp_forward: bad argument");
    cudaStream_t s = nullptr;
    Buf b;
    DevNet d{};
    cudaError_t e = mlp_prepare();
    if (!e) e = upload_net(b, params, norm, d, s);
    float* dX = b.get<float>((size_t)n * kIn);
    float* dY = b.get<float>((size_t)n * kOut);
    int* derr = b.get<int>(1);
    if (!e) e = b.err;
    if (!e) e = cudaMemcpyAsync(dX, X, sizeof(float) * n * kIn, cudaMemcpyHostToDevice, s);
    if (!e) e = cudaMemsetAsync(derr, 0, sizeof(int), s);
    MlpArgs a{};
    a.net = d.view();
    a.n = (int)n;
    a.x = dX;
    a.y = dY;
    a.error = derr;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (!e) e = launch_mlp_forward(a, kModeRaw, sms, s);
    int herr = 0;
    if (!e) e = cudaMemcpyAsync(Y, dY, sizeof(float) * n * kOut, cudaMemcpyDeviceToHost, s);
    if (!e) e = cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (!e) e = cudaStreamSynchronize(s);
    if (e) return mfail(TITAN_ECUDA, std::string("titan_mlp_forward: ") + cudaGetErrorString(e));
    if (herr) return mfail(TITAN_ETIMEOUT, "titan_mlp_forward: a tensor-core wait ran out");
    return TITAN_OK;
}

int titan_mlp_grad(const float* params, const float* norm, const float* X, const float* T, const float* w,
                   const float* row_w, int64_t n, float* grad, float* loss, float* Yout) {
    if (!params || !norm || !X || !T || !w || !grad || n <= 0) return mfail(TITAN_EINVAL, "titan_mlp_grad: bad argument");
    cudaStream_t s = nullptr;
    Buf b;
    Trainer t{};
    if (!alloc_trainer(b, t, (int)n)) return mfail(TITAN_ENOMEM, "titan_mlp_grad: device memory");
    float* dP = b.get<float>(kNParam);
    float* dX = b.get<float>((size_t)n * kIn);
    float* dT = b.get<float>((size_t)n * kOut);
    float* dw = b.get<float>(kOut);
    float* dnorm = b.get<float>(2 * kIn + kOut);
    float* drw = row_w ? b.get<float>((size_t)n) : nullptr;
    if (b.err) return mfail(TITAN_ENOMEM, "titan_mlp_grad: device memory");
    cudaError_t e = cudaMemcpyAsync(dP, params, sizeof(float) * kNParam, cudaMemcpyHostToDevice, s);
    if (!e) e = cudaMemcpyAsync(dX, X, sizeof(float) * n * kIn, cudaMemcpyHostToDevice, s);
    if (!e) e = cudaMemcpyAsync(dT, T, sizeof(float) * n * kOut, cudaMemcpyHostToDevice, s);
    if (!e) e = cudaMemcpyAsync(dw, w, sizeof(float) * kOut, cudaMemcpyHostToDevice, s);
    if (!e) e = cudaMemcpyAsync(dnorm, norm, sizeof(float) * (2 * kIn + kOut), cudaMemcpyHostToDevice, s);
    if (!e && drw) e = cudaMemcpyAsync(drw, row_w, sizeof(float) * n, cudaMemcpyHostToDevice, s);
    if (!e) e = launch_input(dX, dnorm, dnorm + kIn, t.X0, (int)n, s);
    if (!e) e = forward(t, dP, s);
    if (!e) e = backward(t, dT, dw, drw, s);
    if (!e) e = cudaMemcpyAsync(grad, t.grad, sizeof(float) * kNParam, cudaMemcpyDeviceToHost, s);
    if (!e && loss) e = cudaMemcpyAsync(loss, t.loss, sizeof(float), cudaMemcpyDeviceToHost, s);
    if (!e && Yout) e = cudaMemcpy2DAsync(Yout, sizeof(float) * kOut, t.Z[4], sizeof(float) * kOutPad,
                                         sizeof(float) * kOut, n, cudaMemcpyDeviceToHost, s);
    if (!e) e = cudaStreamSynchronize(s);
    if (e) return mfail(TITAN_ECUDA, std::string("titan_mlp_grad: ") + cudaGetErrorString(e));
    if (gemm_error_take()) return mfail(TITAN_ETIMEOUT, "titan_mlp_grad: a tensor-core wait ran out");
    return TITAN_OK;
}

int titan_mlp_train(float* params, const float* norm, const float* X, const float* T, const float* w,
                    const float* row_w, int64_t n, const titan_mlp_train_opts* o, float* loss_per_epoch) {
    if (!params || !norm || !X || !T || !w || !o || n <= 0 || o->batch <= 0 || o->epochs <= 0)
        return mfail(TITAN_EINVAL, "titan_mlp_train: bad argument");
    cudaStream_t s = nullptr;
    const int B = (int)std::min<int64_t>(o->batch, n);
    Buf b;
    Trainer t{};
    if (!alloc_trainer(b, t, B)) return mfail(TITAN_ENOMEM, "titan_mlp_train: device memory");
    float* dP = b.get<float>(kNParam);
    float* dm = b.get<float>(kNParam);
    float* dv = b.get<float>(kNParam);
    unsigned char* dmask = b.get<unsigned char>(kNParam);
    float* dX = b.get<float>((size_t)n * kIn);
    float* dT = b.get<float>((size_t)n * kOut);
    float* dw = b.get<float>(kOut);
    float* dnorm = b.get<float>(2 * kIn + kOut);
    float* drw = row_w ? b.get<float>((size_t)n) : nullptr;
    const int64_t nb = n / B;  // full batches per epoch (rows are pre-shuffled by the caller)
    // the schedule of every step: which batch, and Adam's scalars
    std::vector<TrainSched> sched;
    sched.reserve((size_t)(nb * o->epochs));
    long long step = 0;
    for (int ep = 0; ep < o->epochs; ++ep)
        for (int64_t bi = 0; bi < nb; ++bi) {
            ++step;
            TrainSched q;
            q.r0 = ((bi + (int64_t)ep * 7919) % nb) * B;
            q.c1 = 1.0f - std::pow(o->beta1, (float)step);
            q.c2 = 1.0f - std::pow(o->beta2, (float)step);
            q.lr = o->lr * (o->lr_decay > 0.0f ? std::pow(o->lr_decay, (float)ep) : 1.0f);
            q.epoch = ep;
            sched.push_back(q);
        }
    TrainSched* dS = b.get<TrainSched>(sched.size() + 1);
    int* dstep = b.get<int>(1);
    float* dloss = b.get<float>((size_t)o->epochs);
    if (b.err) return mfail(TITAN_ENOMEM, "titan_mlp_train: device memory");
    // a stream of its own: the batch is captured into a graph from it
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess)
        return mfail(TITAN_ECUDA, "titan_mlp_train: stream");
    const std::vector<unsigned char> mask = param_mask();
    cudaError_t e = cudaMemcpyAsync(dP, params, sizeof(float) * kNParam, cudaMemcpyHostToDevice, s);
    if (!e) e = cudaMemsetAsync(dm, 0, sizeof(float) * kNParam, s);
    if (!e) e = cudaMemsetAsync(dv, 0, sizeof(float) * kNParam, s);
    if (!e) e = cudaMemcpyAsync(dmask, mask.data(), kNParam, cudaMemcpyHostToDevice, s);
    if (!e) e = cudaMemcpyAsync(dX, X, sizeof(float) * n * kIn, cudaMemcpyHostToDevice, s);
    if (!e) e = cudaMemcpyAsync(dT, T, sizeof(float) * n * kOut, cudaMemcpyHostToDevice, s);
    if (!e) e = cudaMemcpyAsync(dw, w, sizeof(float) * kOut, cudaMemcpyHostToDevice, s);
    if (!e) e = cudaMemcpyAsync(dnorm, norm, sizeof(float) * (2 * kIn + kOut), cudaMemcpyHostToDevice, s);
    if (!e && drw) e = cudaMemcpyAsync(drw, row_w, sizeof(float) * n, cudaMemcpyHostToDevice, s);
    if (!e && !sched.empty())
        e = cudaMemcpyAsync(dS, sched.data(), sizeof(TrainSched) * sched.size(), cudaMemcpyHostToDevice, s);
    if (!e) e = cudaMemsetAsync(dstep, 0, sizeof(int), s);
    if (!e) e = cudaMemsetAsync(dloss, 0, sizeof(float) * o->epochs, s);
    // one batch captured once and replayed for every step
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    if (!e && !sched.empty()) {
        e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
        if (!e) {
            cudaError_t ec = launch_input_sched(dX, dnorm, dnorm + kIn, t.X0, B, dS, dstep, s);
            if (!ec) ec = forward(t, dP, s);
            if (!ec) ec = backward_with(t, [&] {
                return launch_loss_sched(t.Z[4], dT, dw, drw, t.rows, t.dY, dloss, dS, dstep, s);
            }, s);
            if (!ec) ec = launch_adam_sched(dP, t.grad, dm, dv, kNParam, o->beta1, o->beta2, 1e-8f, dmask, dS, dstep, s);
            e = cudaStreamEndCapture(s, &g);
            if (!e) e = ec;
        }
        if (!e) e = cudaGraphInstantiate(&ge, g, 0);
        for (size_t k = 0; k < sched.size() && !e; ++k) e = cudaGraphLaunch(ge, s);
    }
    std::vector<float> el((size_t)o->epochs, 0.0f);
    if (!e) e = cudaMemcpyAsync(el.data(), dloss, sizeof(float) * o->epochs, cudaMemcpyDeviceToHost, s);
    if (!e) e = cudaMemcpyAsync(params, dP, sizeof(float) * kNParam, cudaMemcpyDeviceToHost, s);
    if (!e) e = cudaStreamSynchronize(s);
    if (ge) cudaGraphExecDestroy(ge);
    if (g) cudaGraphDestroy(g);
    if (s) cudaStreamDestroy(s);
    if (e) return mfail(TITAN_ECUDA, std::string("titan_mlp_train: ") + cudaGetErrorString(e));
    if (gemm_error_take()) return mfail(TITAN_ETIMEOUT, "titan_mlp_train: a tensor-core wait ran out");
    if (loss_per_epoch)
        for (int ep = 0; ep < o->epochs; ++ep) loss_per_epoch[ep] = el[ep] / (float)(nb > 0 ? nb : 1);
    return TITAN_OK;
}

}  // extern "C"
