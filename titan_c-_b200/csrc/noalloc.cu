// titan_step_noalloc: one plasma step on caller-owned device arrays, with the
// step's scratch (the per-face flux buffer and the status word) in a
// fixed-size array compiled into this library instead of memory it allocates.
//
// Why: some callers cannot call cudaMalloc at the point where they step the
// plasma — a code whose allocator owns all device memory (a framework's
// caching allocator, a memory pool sized at start-up), a real-time loop that
// forbids allocation after initialisation, or an embedding that must not
// touch the CUDA allocator at all. They hand over device pointers they
// already own; this entry point allocates nothing (no cudaMalloc, cudaFree or
// allocating library routine). The same kernels as titan_step run on it.
//
// Limits: a stationary mesh (no node motion) of at most
// TITAN_NOALLOC_MAX_FACES faces. The scratch array lives in every GPU that
// loads the library until the process exits. All calls share it, so calls
// that overlap on the GPU (different streams or threads at the same time)
// race; the array keeps the previous call's contents, and each call resets
// the status word it needs zeroed before its kernels run.
#include <cuda.h>
#include <cuda_runtime.h>

#include <climits>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/titan_b200.h"
#include "launch.h"

namespace titan {
void set_last_error(const std::string& msg);  // titan_api.cu
}

using namespace titan;

namespace {

constexpr size_t kStatusBytes = 256;                       // DevStatus, padded
constexpr size_t kFluxBytesPerFace = 12 * sizeof(double);  // widest flux record (FP64 + Q, rho_He)
constexpr size_t kScratchBytes = kStatusBytes + (size_t)TITAN_NOALLOC_MAX_FACES * kFluxBytesPerFace;
static_assert(sizeof(DevStatus) <= kStatusBytes, "status word must fit its slot");

// The scratch. In host code this name is only a stand-in for the symbol; the
// device address comes from cudaGetSymbolAddress (see scratch_on_device).
__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

int nfail(int code, const std::string& msg) {
    titan::set_last_error(msg);  // reported by titan_last_error()
    return code;
}

// Device address of the scratch on the current device, looked up with that
// device current and cached together with the context it belongs to. A device
// reset (cudaDeviceReset) destroys the context and the module with the array;
// the next call then sees a different current context and looks the address
// up again instead of using the stale one. The current context comes from the
// driver's cuCtxGetCurrent, fetched through the runtime (no libcuda link).
using CtxGetCurrentFn = CUresult (*)(CUcontext*);
std::mutex g_mu;
void* g_addr[256] = {};
CUcontext g_ctx[256] = {};
CtxGetCurrentFn g_ctx_get = nullptr;

int scratch_on_device(unsigned char** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 256) return nfail(TITAN_ECUDA, "titan_step_noalloc: no current device");
    e = cudaSetDevice(dev);  // makes the device's primary context current on this thread
    if (e != cudaSuccess)
        return nfail(TITAN_ECUDA, std::string("titan_step_noalloc: no context: ") + cudaGetErrorString(e));
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_ctx_get) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q);
        if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn)
            return nfail(TITAN_ECUDA, "titan_step_noalloc: cuCtxGetCurrent not available");
        g_ctx_get = reinterpret_cast<CtxGetCurrentFn>(fn);
    }
    CUcontext ctx = nullptr;
    if (g_ctx_get(&ctx) != CUDA_SUCCESS || !ctx) return nfail(TITAN_ECUDA, "titan_step_noalloc: no current context");
    if (!g_addr[dev] || g_ctx[dev] != ctx) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return nfail(TITAN_ECUDA, std::string("titan_step_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_addr[dev] = p;
        g_ctx[dev] = ctx;
    }
    *out = static_cast<unsigned char*>(g_addr[dev]);
    return TITAN_OK;
}

__global__ void noalloc_reset_status(DevStatus* st, double dt) {
    st->err_kind = 0;
    st->err_index = 0;
    st->n_rho_floor = 0;
    st->n_p_floor = 0;
    st->steps_done = 0;
    st->block_counter = 0;
    st->dt_next_bits = 0x4197D78400000000ull;  // bits of 1e8, identity of the CFL minimum
    st->dt = dt;
    st->t = 0.0;
}

}  // namespace

extern "C" int titan_step_noalloc(const titan_dev_mesh* m, const titan_params* p, double dt, const double* state_in,
                                  double* state_out, double* dt_next, int32_t* err_kind, void* stream) {
    if (!m || !p || !state_in || !state_out || !dt_next) return nfail(TITAN_EINVAL, "titan_step_noalloc: null argument");
    if (m->nface <= 0 || m->ncell <= 0) return nfail(TITAN_EINVAL, "titan_step_noalloc: empty mesh");
    // every cell lists 6 faces and a face belongs to at most 2 cells, so
    // 3 ncell <= nface; this also keeps ncell far inside the kernels' int range
    if (m->ncell > INT_MAX / 3 || 3 * m->ncell > m->nface)
        return nfail(TITAN_EINVAL, "titan_step_noalloc: ncell inconsistent with nface (6 faces per cell, 2 cells per face)");
    if (m->nbc < 0 || m->nbc > INT_MAX) return nfail(TITAN_EINVAL, "titan_step_noalloc: nbc out of range");
    if (m->nface > TITAN_NOALLOC_MAX_FACES) {
        char buf[200];
        snprintf(buf, sizeof buf, "titan_step_noalloc: %lld faces exceed the fixed scratch of %d faces",
                 (long long)m->nface, (int)TITAN_NOALLOC_MAX_FACES);
        return nfail(TITAN_EINVAL, buf);
    }
    if (p->move) return nfail(TITAN_EINVAL, "titan_step_noalloc: stationary meshes only (move = 0)");
    if (p->tvd) return nfail(TITAN_EINVAL, "titan_step_noalloc: first-order faces only (tvd = 0)");
    if (p->bn_in_p_on_hp) return nfail(TITAN_EINVAL, "titan_step_noalloc: no exact HP solver (bn_in_p_on_hp = 0)");
    if (p->npassive != 0 && p->npassive != 2) return nfail(TITAN_EINVAL, "titan_step_noalloc: npassive must be 0 or 2");
    if (p->flux_precision != 64 && p->flux_precision != 32)
        return nfail(TITAN_EINVAL, "titan_step_noalloc: flux_precision must be 64 or 32");
    if (p->nh < 0 || p->nh > 4 || (p->nh > 0 && !m->hfluids))
        return nfail(TITAN_EINVAL, "titan_step_noalloc: nh must be 0..4 and needs hfluids");
    if (!(dt > 0.0)) return nfail(TITAN_EINVAL, "titan_step_noalloc: dt must be positive");

    unsigned char* scratch = nullptr;
    int rc = scratch_on_device(&scratch);
    if (rc) return rc;
    DevStatus* st = reinterpret_cast<DevStatus*>(scratch);
    void* flux = scratch + kStatusBytes;
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    MeshView M{};
    M.ncell = (int)m->ncell;
    M.nface = (int)m->nface;
    M.nnode = 0;
    M.nbc = (int)m->nbc;
    M.face_c0 = m->face_c0;
    M.face_c1 = m->face_c1;
    M.face_type = m->face_type;
    M.face_surf = m->face_surf;
    M.face_method = m->face_method;
    M.face_bc = m->face_bc;
    M.bc_vals = m->bc_vals;
    M.cell_faces = m->cell_faces;
    M.cell_type = m->cell_type;
    M.cell_tvd = m->cell_tvd;
    Layer L{};
    L.cc = const_cast<double*>(m->cell_center);
    L.vol = const_cast<double*>(m->cell_volume);
    L.fc = const_cast<double*>(m->face_center);
    L.fn = const_cast<double*>(m->face_normal);
    L.fa = const_cast<double*>(m->face_area);
    L.fd = const_cast<double*>(m->face_half_dist);
    Params P{};
    P.gamma = p->gamma;
    P.KFL = p->KFL;
    P.velosity_inf = p->velosity_inf;
    P.omega = p->omega;
    P.par_a_2 = p->par_a_2;
    P.par_n_H_LISM = p->par_n_H_LISM;
    P.par_Kn = p->par_Kn;
    P.beta_switch = p->beta_switch;
    P.soft_fixups = p->soft_fixups;
    P.method_policy = p->method_policy;
    P.npassive = p->npassive;
    P.nh = p->nh;
    P.TS_hard = p->TS_hard;
    P.contact_hard = p->contact_hard;

    (void)cudaGetLastError();
    noalloc_reset_status<<<1, 1, 0, s>>>(st, dt);
    cudaError_t e = cudaGetLastError();
    FaceArgs fa{};
    fa.M = M;
    fa.P = P;
    fa.L1 = L;
    fa.xyz2 = nullptr;
    fa.state = state_in;
    fa.flux = flux;
    fa.st = st;
    const bool fp32 = p->flux_precision == 32;
    if (!e) e = fp32 ? launch_face_flux_fp32(fa, p->npassive, false, 0, s) : launch_face_flux_fp64(fa, p->npassive, false, 0, s);
    CellArgs ca{};
    ca.M = M;
    ca.P = P;
    ca.vol1 = m->cell_volume;
    ca.vol2 = m->cell_volume;
    ca.state = state_in;
    ca.state2 = state_out;
    ca.flux = flux;
    ca.hfl = m->hfluids;
    ca.src = nullptr;
    ca.st = st;
    if (!e) e = launch_cell_update(ca, p->npassive, false, p->nh > 0 ? 1 : 0, 0, s);
    DevStatus h{};
    if (!e) e = cudaMemcpyAsync(&h, st, sizeof(DevStatus), cudaMemcpyDeviceToHost, s);
    if (!e) e = cudaStreamSynchronize(s);
    if (e) return nfail(TITAN_ECUDA, std::string("titan_step_noalloc: ") + cudaGetErrorString(e));
    *dt_next = h.dt;
    if (err_kind) *err_kind = h.err_kind;
    if (h.err_kind != 0) {
        char buf[160];
        snprintf(buf, sizeof buf, "titan_step_noalloc: step failed, kind %d at index %d", h.err_kind, h.err_index);
        return nfail(h.err_kind >= 20 ? TITAN_ENONFINITE : TITAN_ESOLVER, buf);
    }
    return TITAN_OK;
}
