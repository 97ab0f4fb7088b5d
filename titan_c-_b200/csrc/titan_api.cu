// Host side of the C ABI declared in include/titan_b200.h: mesh validation and
// SFC renumbering, device buffers, the step loop (CUDA-graph captured), and
// the state / geometry / flux transfers in the caller's original numbering.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <array>
#include <map>
#include <tuple>
#include <string>
#include <vector>

#include "../../include/titan_b200.h"
#include "closure.h"
#include "halo.h"
#include "launch.h"
#include "mc.h"
#include "renumber.h"
#include "surface.h"

using namespace titan;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

#define CK(call)                                                                                     \
    do {                                                                                             \
        cudaError_t e_ = (call);                                                                     \
        if (e_ != cudaSuccess)                                                                       \
            return fail(e_ == cudaErrorMemoryAllocation ? TITAN_ENOMEM : TITAN_ECUDA,                \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                         \
    } while (0)

template <typename T>
cudaError_t dalloc(T** p, size_t n, int64_t* total) {
    *p = nullptr;
    if (n == 0) return cudaSuccess;
    *total += int64_t(n * sizeof(T));
    return cudaMalloc((void**)p, n * sizeof(T));
}

template <typename T>
cudaError_t dput(T* d, const std::vector<T>& h, cudaStream_t s) {
    if (h.empty()) return cudaSuccess;
    return cudaMemcpyAsync(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, s);
}

}  // namespace

namespace titan {
// Lets other translation units report through titan_last_error().
void set_last_error(const std::string& msg) { g_err = msg; }
}  // namespace titan

struct KernelClock {
    double ms = 0.0;
    int64_t launches = 0;
};

struct titan_ctx {
    int64_t ncell = 0, nface = 0, nnode = 0, nbc = 0;
    titan_params prm{};
    Params P{};
    int ns = 8;  // state fields stored on the device (8 + npassive)
    bool fp32 = false;
    cudaStream_t stream = nullptr;
    // the closure's own stream (the greatest priority), forked from and joined
    // back into `stream` so the network runs beside the face kernel
    cudaStream_t side = nullptr;
    cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
    bool overlap_closure = true;
    int64_t dev_bytes = 0;

    Renumbering R;
    int32_t* d_cell_n2o = nullptr;
    int32_t* d_node_n2o = nullptr;

    // mesh (renumbered)
    int32_t *d_face_c0 = nullptr, *d_face_c1 = nullptr, *d_face_bc = nullptr, *d_face_nodes = nullptr;
    int8_t *d_face_type = nullptr, *d_face_surf = nullptr, *d_face_method = nullptr;
    double* d_bc_vals = nullptr;
    int32_t *d_cell_faces = nullptr, *d_cell_nodes = nullptr;
    int32_t* d_owner_start = nullptr;  // [ceil(ncell/32)+1] first face owned by each 32-cell chunk
    int8_t* d_cell_type = nullptr;
    uint8_t* d_cell_tvd = nullptr;
    double *d_node_amp = nullptr, *d_node_phase = nullptr;
    uint16_t* d_cell_fmap = nullptr;
    int32_t *d_face_aa = nullptr, *d_face_bb = nullptr;  // second-order neighbours (tvd)

    Layer layer[2]{};
    int cur = 0;
    double* d_state[2] = {nullptr, nullptr};
    int scur = 0;
    void* d_flux = nullptr;
    int flux_stride = 0;
    size_t flux_elem = 8;
    double* d_hfl = nullptr;
    double* d_src = nullptr;
    bool use_src = false;
    double* d_stage = nullptr;  // NV*max(ncell, nnode) staging for transfers
    DevStatus* d_status = nullptr;
    DevStatus* h_status = nullptr;  // pinned

    // CUDA graph of two steps (the buffer ping-pong has period two)
    cudaGraphExec_t graph = nullptr;
    int graph_cur = -1, graph_scur = -1;

    ClosureDev closure;        // learned sources (titan_set_closure)
    bool use_closure = false;
    uint32_t* d_cl_in = nullptr;        // [8][ncell] the network's input words for the next step
    float* d_cl_y = nullptr;            // [5][ncell] the network's outputs of the current step
    unsigned char* d_cl_out = nullptr;  // [ncell] the next step's cells outside the training envelope
    bool cl_valid = false;              // d_cl_in / d_cl_out match the current state and centres
    float* d_env = nullptr;    // [2][8] training envelope (titan_set_closure_fallback)
    double* d_fallback = nullptr;       // [4][ncell] fallback sources, renumbered
    unsigned long long* d_n_outside = nullptr;
    double closure_ninf = 0.0, closure_lambda = 0.0;
    int sm_count = 148;

    signed char* d_face_nodt = nullptr;  // faces left out of the CFL minimum (titan_set_cfl_faces)

    // halo exchange of a sharded step (titan_set_halo): renumbered cell ids
    int32_t* d_halo_send = nullptr;
    int32_t* d_halo_recv = nullptr;
    int64_t n_halo_send = 0, n_halo_recv = 0;

    // surface-tracking node motion (titan_set_surface_motion)
    bool use_surface = false;
    SurfaceDev surf{};
    std::vector<int32_t> h_ray_nodes;  // the rays of surf (device node ids, -1 padding)
    std::vector<int8_t> h_node_surf;   // per device node: the surface (1 TS, 2 HP, 3 BS) it lies on, or 0
    void* surf_buf[15] = {};  // face_list, vf, node_id, node_ptr, node_face, ray_nodes, ray_r0, ray_dir, ray_seg,
                              // sm_kind, sm_coef, sm_centre, nb_ptr, nb_id

    // Monte-Carlo pass buffers (titan_mc_sources), allocated by the first pass
    McCell* d_mc_cells = nullptr;       // [ncell] tracing records
    double* d_mc_cdf = nullptr;         // [nface] inflow CDF
    // tabulated inflow distributions (titan_set_mc_face_dist): index, frame,
    // side, flux, leaf_ptr, box, cum (McFaceDist)
    void* fd_buf[7] = {};
    // tallied outgoing distributions (titan_set_mc_face_tally): index, face,
    // side, frame, bounds, leaf_ptr, box, f, mom, unplaced (McFaceTally)
    void* ft_buf[10] = {};
    int64_t ft_ntab = 0, ft_nleaf = 0;
    bool ft_valid = false;  // the tables hold a finished pass
    double* d_mc_blocks = nullptr;      // [mc_scan_blocks(nface)] + 1: block sums, total
    double* d_mc_tally = nullptr;       // [5][ncell]
    unsigned long long* d_mc_lost = nullptr;
    bool mc_valid = false;              // d_mc_tally holds a finished pass

    int face_variant = 0;  // launch shapes (autotuned, see titan_autotune)
    int cell_variant = 0;

    bool profiling = false;
    std::map<std::string, KernelClock> clocks;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    // state transfers: copies on their own stream, one event per field, so the
    // copy of one field overlaps the renumbering of another
    cudaStream_t xfer = nullptr;
    cudaEvent_t xev[TITAN_NV + 1] = {};

    MeshView view() const {
        MeshView M;
        M.ncell = (int)ncell;
        M.nface = (int)nface;
        M.nnode = (int)nnode;
        M.nbc = (int)nbc;
        M.face_c0 = d_face_c0;
        M.face_c1 = d_face_c1;
        M.face_type = d_face_type;
        M.face_surf = d_face_surf;
        M.face_method = d_face_method;
        M.face_bc = d_face_bc;
        M.bc_vals = d_bc_vals;
        M.face_nodes = d_face_nodes;
        M.cell_faces = d_cell_faces;
        M.cell_nodes = d_cell_nodes;
        M.cell_type = d_cell_type;
        M.cell_tvd = d_cell_tvd;
        M.node_amp = d_node_amp;
        M.node_phase = d_node_phase;
        M.cell_fmap = d_cell_fmap;
        M.face_aa = d_face_aa;
        M.face_bb = d_face_bb;
        M.face_nodt = d_face_nodt;
        return M;
    }
};

namespace {

// Runs `fn` (which launches one kernel on ctx->stream); when profiling, times
// it with CUDA events under `name`.
template <typename F>
cudaError_t timed(titan_ctx* ctx, const char* name, F fn) {
    if (!ctx->profiling) return fn();
    cudaEventRecord(ctx->ev[0], ctx->stream);
    cudaError_t e = fn();
    cudaEventRecord(ctx->ev[1], ctx->stream);
    cudaEventSynchronize(ctx->ev[1]);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
    KernelClock& k = ctx->clocks[name];
    k.ms += ms;
    k.launches += 1;
    return e;
}

// The face-flux kernel of this context: FP64 or FP32 Riemann arithmetic,
// first- or second-order faces.
cudaError_t face_launch(const titan_ctx* ctx, const FaceArgs& fa, int nk, bool move, int variant, cudaStream_t s) {
    if (ctx->P.tvd)
        return ctx->fp32 ? launch_face_flux_tvd_fp32(fa, nk, move, variant, s)
                         : launch_face_flux_tvd_fp64(fa, nk, move, variant, s);
    return ctx->fp32 ? launch_face_flux_fp32(fa, nk, move, variant, s) : launch_face_flux_fp64(fa, nk, move, variant, s);
}

const char* face_kernel_name(const titan_ctx* ctx) {
    if (ctx->P.tvd) return ctx->fp32 ? "face_flux_tvd_fp32" : "face_flux_tvd_fp64";
    return ctx->fp32 ? "face_flux_fp32" : "face_flux_fp64";
}

// The closure's part of the cell update (source mode 3) for the current buffers.
ClosureCell closure_cell(const titan_ctx* ctx) {
    ClosureCell q{};
    q.y = ctx->d_cl_y;
    q.in = ctx->d_cl_in;
    q.outside = ctx->d_cl_out;
    q.fallback = ctx->d_fallback;
    q.n_outside = ctx->d_n_outside;
    q.norm = ctx->closure.norm;
    q.env = ctx->d_env;
    q.nH_inf = ctx->closure_ninf;
    q.lambda = ctx->closure_lambda;
    q.cc1 = ctx->layer[ctx->cur].cc;
    return q;
}

int step_source_mode(const titan_ctx* ctx) {
    return ctx->use_closure ? 3 : (ctx->use_src ? 2 : (ctx->prm.nh > 0 ? 1 : 0));
}

// Enqueue one step; flips the layer and state buffers.
cudaError_t enqueue_step(titan_ctx* ctx) {
    const MeshView M = ctx->view();
    const bool move = ctx->prm.move != 0;
    const bool overlap = ctx->use_closure && ctx->overlap_closure && !ctx->profiling;
    const int nxt = ctx->cur ^ 1;
    cudaError_t e = cudaSuccess;
    if (ctx->use_closure) {
        // the network on this step's inputs (formed by the previous cell update);
        // the cell update turns its outputs into sources. It reads neither the
        // nodes nor the state, so it starts before the node motion.
        MlpArgs ma{};
        ma.net = ctx->closure.view();
        ma.n = (int)ctx->ncell;
        ma.ncell = (int)ctx->ncell;
        ma.in_words = ctx->d_cl_in;
        ma.y_out = ctx->d_cl_y;
        ma.error = ctx->closure.error;
        if (ctx->d_n_outside) {
            e = cudaMemsetAsync(ctx->d_n_outside, 0, sizeof(unsigned long long), ctx->stream);
            if (e) return e;
        }
        if (overlap) {
            // beside the node motion and the face kernel; the cell update waits
            // for it (kernel-time profiling keeps the kernels in turn)
            e = cudaEventRecord(ctx->fork_ev, ctx->stream);
            if (!e) e = cudaStreamWaitEvent(ctx->side, ctx->fork_ev, 0);
            if (!e) e = launch_mlp_forward(ma, kModeSources, ctx->sm_count, ctx->side);
            if (!e) e = cudaEventRecord(ctx->join_ev, ctx->side);
        } else {
            e = timed(ctx, "closure_mlp",
                      [&] { return launch_mlp_forward(ma, kModeSources, ctx->sm_count, ctx->stream); });
        }
        if (e) return e;
    }
    if (move && ctx->use_surface) {
        // nodes follow the TS / HP / BS surfaces (Setka::Culc_Velocity_surface,
        // Luch::dvigenie) on this state; null_bn_on_HP may edit the HP cells' B
        FaceArgs sa;
        sa.M = M;
        sa.P = ctx->P;
        sa.L1 = ctx->layer[ctx->cur];
        sa.xyz2 = ctx->layer[nxt].xyz;
        sa.state = ctx->d_state[ctx->scur];
        sa.flux = nullptr;
        sa.st = ctx->d_status;
        e = timed(ctx, "surface_motion", [&] {
            return launch_surface_motion(sa, ctx->d_state[ctx->scur], ctx->surf, ctx->prm.npassive, ctx->P.tvd != 0,
                                         ctx->stream);
        });
        if (e) return e;
    } else if (move) {
        // the geometry of the next layer is formed inside face_flux (faces of
        // this layer) and cell_update (cells of the next layer)
        e = timed(ctx, "move_nodes", [&] {
            return launch_move_nodes(M, ctx->P, ctx->layer[ctx->cur].xyz, ctx->layer[nxt].xyz, ctx->d_status,
                                     ctx->stream);
        });
        if (e) return e;
    }
    FaceArgs fa;
    fa.M = M;
    fa.P = ctx->P;
    fa.L1 = ctx->layer[ctx->cur];
    fa.xyz2 = move ? ctx->layer[nxt].xyz : ctx->layer[ctx->cur].xyz;
    fa.state = ctx->d_state[ctx->scur];
    fa.flux = ctx->d_flux;
    fa.st = ctx->d_status;
    const int nk = ctx->prm.npassive;
    e = timed(ctx, face_kernel_name(ctx), [&] { return face_launch(ctx, fa, nk, move, ctx->face_variant, ctx->stream); });
    if (!e && overlap) e = cudaStreamWaitEvent(ctx->stream, ctx->join_ev, 0);
    if (e) return e;
    CellArgs ca;
    ca.M = M;
    ca.P = ctx->P;
    ca.vol1 = ctx->layer[ctx->cur].vol;
    ca.vol2 = ctx->layer[ctx->cur].vol;
    ca.L2 = ctx->layer[nxt];
    ca.state = ctx->d_state[ctx->scur];
    ca.state2 = ctx->d_state[ctx->scur ^ 1];
    ca.flux = ctx->d_flux;
    ca.hfl = ctx->d_hfl;
    ca.src = ctx->d_src;
    ca.cl = closure_cell(ctx);
    ca.st = ctx->d_status;
    ca.owner_start = ctx->d_owner_start;
    const int src = step_source_mode(ctx);
    e = timed(ctx, "cell_update",
              [&] { return launch_cell_update(ca, nk, move, src, ctx->cell_variant, ctx->stream); });
    if (e) return e;
    ctx->scur ^= 1;
    if (move) ctx->cur = nxt;
    return cudaSuccess;
}

void drop_graph(titan_ctx* ctx) {
    if (ctx->graph) cudaGraphExecDestroy(ctx->graph);
    ctx->graph = nullptr;
    ctx->graph_cur = ctx->graph_scur = -1;
}

// Captures two steps into a CUDA graph starting from the current buffer phase.
cudaError_t capture_two_steps(titan_ctx* ctx) {
    drop_graph(ctx);
    const int c0 = ctx->cur, s0 = ctx->scur;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
    if (e) return e;
    cudaError_t e1 = enqueue_step(ctx);
    cudaError_t e2 = e1 ? e1 : enqueue_step(ctx);
    e = cudaStreamEndCapture(ctx->stream, &g);
    ctx->cur = c0;
    ctx->scur = s0;
    if (e2) {
        if (g) cudaGraphDestroy(g);
        return e2;
    }
    if (e) return e;
    e = cudaGraphInstantiate(&ctx->graph, g, 0);
    cudaGraphDestroy(g);
    if (e) return e;
    ctx->graph_cur = c0;
    ctx->graph_scur = s0;
    return cudaSuccess;
}

std::string validate(const titan_mesh* m, const titan_params* p) {
    char buf[256];
    if (m->ncell <= 0 || m->nface <= 0 || m->nnode <= 0) return "empty mesh";
    if (m->ncell >= (1LL << 31) - 1 || m->nface >= (1LL << 31) - 1 || m->nnode >= (1LL << 31) - 1)
        return "mesh too large for 32-bit indices";
    if (!m->node_xyz || !m->cell_nodes || !m->cell_faces || !m->cell_type || !m->cell_tvd || !m->face_nodes ||
        !m->face_cells || !m->face_type || !m->face_surf || !m->face_bc)
        return "null mesh array";
    if ((m->node_amp == nullptr) != (m->node_phase == nullptr)) return "node_amp and node_phase go together";
    if (p->move && !m->node_amp) return "move requires node_amp / node_phase";
    if (p->npassive != 0 && p->npassive != 2) return "npassive must be 0 or 2";
    if (p->nh < 0 || p->nh > 4) return "nh must be 0..4";
    if (p->flux_precision != 64 && p->flux_precision != 32) return "flux_precision must be 64 or 32";
    if (p->tvd != 0 && p->tvd != 1) return "tvd must be 0 or 1";
    if (!(p->gamma > 1.0)) return "gamma must exceed 1";
    for (int64_t i = 0; i < 3 * m->nnode; ++i)
        if (!std::isfinite(m->node_xyz[i])) return "non-finite node coordinate";
    for (int64_t c = 0; c < m->ncell; ++c) {
        for (int k = 0; k < 8; ++k) {
            const int32_t v = m->cell_nodes[8 * c + k];
            if (v < 0 || v >= m->nnode) {
                snprintf(buf, sizeof buf, "cell %lld: node index out of range", (long long)c);
                return buf;
            }
        }
        for (int s = 0; s < 6; ++s) {
            const int32_t f = m->cell_faces[6 * c + s];
            if (f < 0 || f >= m->nface) {
                snprintf(buf, sizeof buf, "cell %lld: face index out of range", (long long)c);
                return buf;
            }
            if (m->face_cells[2 * f] != c && m->face_cells[2 * f + 1] != c) {
                snprintf(buf, sizeof buf, "cell %lld lists face %d which does not list it", (long long)c, f);
                return buf;
            }
        }
        if (m->cell_type[c] < 0 || m->cell_type[c] > 4) return "cell_type out of range";
    }
    for (int64_t f = 0; f < m->nface; ++f) {
        for (int k = 0; k < 4; ++k) {
            const int32_t v = m->face_nodes[4 * f + k];
            if (v < 0 || v >= m->nnode) {
                snprintf(buf, sizeof buf, "face %lld: node index out of range", (long long)f);
                return buf;
            }
        }
        const int32_t c0 = m->face_cells[2 * f], c1 = m->face_cells[2 * f + 1];
        const int t = m->face_type[f];
        if (c0 < 0 || c0 >= m->ncell) {
            snprintf(buf, sizeof buf, "face %lld: cells[0] out of range", (long long)f);
            return buf;
        }
        if (t < 0 || t > 3) return "face_type out of range";
        if (m->face_surf[f] < 0 || m->face_surf[f] > 3) return "face_surf out of range";
        if (t == 0 && (c1 < 0 || c1 >= m->ncell)) {
            snprintf(buf, sizeof buf, "interior face %lld needs two cells", (long long)f);
            return buf;
        }
        if (t != 0 && c1 != -1) {
            snprintf(buf, sizeof buf, "boundary face %lld must have one cell", (long long)f);
            return buf;
        }
        if (t == 1 || t == 2) {
            const int32_t r = m->face_bc[f];
            if (r < 0 || r >= m->nbc || !m->bc_vals) {
                snprintf(buf, sizeof buf, "hard boundary face %lld has no fixed values", (long long)f);
                return buf;
            }
        }
    }
    return "";
}

}  // namespace

namespace {

void drop_surface(titan_ctx* ctx) {
    for (void*& p : ctx->surf_buf) {
        if (p) cudaFree(p);
        p = nullptr;
    }
    ctx->surf = SurfaceDev{};
    ctx->use_surface = false;
}

// Least squares of 2 p . c = |p|^2 over the points with weights w (normal
// equations, Gaussian elimination with partial pivoting); a singular system
// (all weights zero) gives the zero vector.
void fit_weighted(const std::vector<std::array<double, 3>>& P, const std::vector<double>& w, double c[3]) {
    double M[3][4] = {};
    for (size_t i = 0; i < P.size(); ++i) {
        const double a[3] = {2.0 * P[i][0], 2.0 * P[i][1], 2.0 * P[i][2]};
        const double b = P[i][0] * P[i][0] + P[i][1] * P[i][1] + P[i][2] * P[i][2];
        const double ww = w[i] * w[i];
        for (int j = 0; j < 3; ++j) {
            for (int k = 0; k < 3; ++k) M[j][k] += ww * a[j] * a[k];
            M[j][3] += ww * a[j] * b;
        }
    }
    double scale = 0.0;
    for (int j = 0; j < 3; ++j)
        for (int k = 0; k < 3; ++k) scale = std::max(scale, std::fabs(M[j][k]));
    c[0] = c[1] = c[2] = 0.0;
    if (!(scale > 0.0)) return;
    for (int col = 0; col < 3; ++col) {
        int piv = col;
        for (int r = col + 1; r < 3; ++r)
            if (std::fabs(M[r][col]) > std::fabs(M[piv][col])) piv = r;
        if (std::fabs(M[piv][col]) <= 1e-14 * scale) return;
        if (piv != col)
            for (int k = 0; k < 4; ++k) std::swap(M[col][k], M[piv][k]);
        for (int r = col + 1; r < 3; ++r) {
            const double f = M[r][col] / M[col][col];
            for (int k = col; k < 4; ++k) M[r][k] -= f * M[col][k];
        }
    }
    for (int j = 2; j >= 0; --j) {
        double v = M[j][3];
        for (int k = j + 1; k < 3; ++k) v -= M[j][k] * c[k];
        c[j] = v / M[j][j];
    }
}

// Centre of the sphere that best fits a node and its surface neighbours, as
// Setka::Smooth_head_TS3 / Smooth_head_HP3 form it (Setka_move.cpp:2205-2362,
// 2046-2203): the least-squares c of 2 p . c = |p|^2, then up to 8 fits
// re-weighted by Tukey's biweight of the distance residuals (cutoff 2.5
// standard deviations), until the RMS residual changes by less than 1e-6.
// The reference solves each fit by SVD; the normal equations here give the
// same centre up to rounding.
void fit_centre(const std::vector<std::array<double, 3>>& P, double c[3]) {
    const size_t n = P.size();
    std::vector<double> w(n, 1.0), res(n);
    fit_weighted(P, w, c);
    double prev = 1e308;
    for (int iter = 0; iter < 8; ++iter) {
        double radius = 0.0;
        for (const auto& p : P)
            radius += std::sqrt((p[0] - c[0]) * (p[0] - c[0]) + (p[1] - c[1]) * (p[1] - c[1]) +
                                (p[2] - c[2]) * (p[2] - c[2]));
        radius /= (double)n;
        double total = 0.0;
        for (size_t i = 0; i < n; ++i) {
            const double d = std::sqrt((P[i][0] - c[0]) * (P[i][0] - c[0]) + (P[i][1] - c[1]) * (P[i][1] - c[1]) +
                                       (P[i][2] - c[2]) * (P[i][2] - c[2]));
            res[i] = std::fabs(d - radius);
            total += res[i] * res[i];
        }
        const double rms = std::sqrt(total / (double)n);
        if (std::fabs(prev - rms) < 1e-6) break;
        prev = rms;
        double mean = 0.0;
        for (double r : res) mean += r;
        mean /= (double)n;
        double var = 0.0;
        for (double r : res) var += (r - mean) * (r - mean);
        const double cutoff = 2.5 * std::sqrt(var / (double)n);
        for (size_t i = 0; i < n; ++i) {
            if (res[i] < cutoff) {
                const double t = res[i] / cutoff;
                w[i] = (1.0 - t * t) * (1.0 - t * t);
            } else {
                w[i] = 0.0;
            }
        }
        fit_weighted(P, w, c);
    }
}

template <typename T>
cudaError_t upload_vec(void** slot, const std::vector<T>& v) {
    if (v.empty()) return cudaSuccess;
    cudaError_t e = cudaMalloc(slot, sizeof(T) * v.size());
    if (!e) e = cudaMemcpy(*slot, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice);
    return e;
}

}  // namespace

extern "C" {

const char* titan_version(void) { return "titan-b200 0.1 (sm_100a)"; }

const char* titan_last_error(void) { return g_err.c_str(); }

int titan_destroy(titan_ctx* ctx) {
    if (!ctx) return TITAN_OK;
    drop_graph(ctx);
    closure_destroy(&ctx->closure);
    void* ptrs[] = {ctx->d_cell_n2o, ctx->d_node_n2o, ctx->d_face_c0, ctx->d_face_c1, ctx->d_face_bc,
                    ctx->d_face_nodes, ctx->d_face_type, ctx->d_face_surf, ctx->d_face_method, ctx->d_bc_vals,
                    ctx->d_cell_faces, ctx->d_cell_nodes, ctx->d_cell_type, ctx->d_cell_tvd, ctx->d_node_amp,
                    ctx->d_node_phase, ctx->d_state[0], ctx->d_state[1], ctx->d_flux, ctx->d_hfl, ctx->d_src,
                    ctx->d_stage, ctx->d_status, ctx->d_cell_fmap, ctx->d_face_aa, ctx->d_face_bb,
                    ctx->d_env, ctx->d_fallback, ctx->d_n_outside, ctx->d_mc_cells, ctx->d_mc_cdf,
                    ctx->d_mc_blocks, ctx->d_mc_tally, ctx->d_mc_lost, ctx->d_owner_start};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    for (void* p : ctx->surf_buf)
        if (p) cudaFree(p);
    for (void* p : ctx->fd_buf)
        if (p) cudaFree(p);
    for (void* p : ctx->ft_buf)
        if (p) cudaFree(p);
    if (ctx->d_cl_in) cudaFree(ctx->d_cl_in);
    if (ctx->d_cl_y) cudaFree(ctx->d_cl_y);
    if (ctx->d_cl_out) cudaFree(ctx->d_cl_out);
    if (ctx->d_halo_send) cudaFree(ctx->d_halo_send);
    if (ctx->d_halo_recv) cudaFree(ctx->d_halo_recv);
    if (ctx->d_face_nodt) cudaFree(ctx->d_face_nodt);
    // without node motion layer[1] aliases layer[0]: free it once
    const int nlayers = (ctx->layer[1].xyz != ctx->layer[0].xyz) ? 2 : 1;
    for (int l = 0; l < nlayers; ++l) {
        Layer& L = ctx->layer[l];
        void* lp[] = {L.xyz, L.cc, L.vol, L.fc, L.fn, L.fa, L.fd};
        for (void* p : lp)
            if (p) cudaFree(p);
    }
    if (ctx->h_status) cudaFreeHost(ctx->h_status);
    for (auto& e : ctx->ev)
        if (e) cudaEventDestroy(e);
    for (auto& e : ctx->xev)
        if (e) cudaEventDestroy(e);
    if (ctx->xfer) cudaStreamDestroy(ctx->xfer);
    if (ctx->side) cudaStreamDestroy(ctx->side);
    if (ctx->fork_ev) cudaEventDestroy(ctx->fork_ev);
    if (ctx->join_ev) cudaEventDestroy(ctx->join_ev);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return TITAN_OK;
}

int titan_create(const titan_mesh* m, const titan_params* p, titan_ctx** out) {
    if (!m || !p || !out) return fail(TITAN_EINVAL, "null argument");
    *out = nullptr;
    const std::string v = validate(m, p);
    if (!v.empty()) return fail(TITAN_EMESH, v);

    (void)cudaGetLastError();  // launch checks below must not see an earlier call's error
    titan_ctx* ctx = new titan_ctx();
    ctx->ncell = m->ncell;
    ctx->nface = m->nface;
    ctx->nnode = m->nnode;
    ctx->nbc = m->nbc;
    ctx->prm = *p;
    ctx->fp32 = p->flux_precision == 32;
    ctx->ns = 8 + p->npassive;
    Params& P = ctx->P;
    P.gamma = p->gamma;
    P.KFL = p->KFL;
    P.velosity_inf = p->velosity_inf;
    P.omega = p->omega;
    P.par_a_2 = p->par_a_2;
    P.par_n_H_LISM = p->par_n_H_LISM;
    P.par_Kn = p->par_Kn;
    P.beta_switch = p->beta_switch;
    P.move = p->move;
    P.soft_fixups = p->soft_fixups;
    P.method_policy = p->method_policy;
    P.npassive = p->npassive;
    P.nh = p->nh;
    P.TS_hard = p->TS_hard;
    P.contact_hard = p->contact_hard;
    P.src_mode = 0;
    P.tvd = p->tvd;
    P.snos_on_hp = p->snos_on_hp;
    P.bn_in_p_on_hp = p->bn_in_p_on_hp;

    auto bail = [&](int code) {
        titan_destroy(ctx);
        return code;
    };
    cudaError_t e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e) return bail(fail(TITAN_ECUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e)));
    cudaEventCreate(&ctx->ev[0]);
    cudaEventCreate(&ctx->ev[1]);
    e = cudaStreamCreateWithFlags(&ctx->xfer, cudaStreamNonBlocking);
    if (e) return bail(fail(TITAN_ECUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e)));
    {
        int lo = 0, hi = 0;
        e = cudaDeviceGetStreamPriorityRange(&lo, &hi);
        if (!e) e = cudaStreamCreateWithPriority(&ctx->side, cudaStreamNonBlocking, hi);
        if (!e) e = cudaEventCreateWithFlags(&ctx->fork_ev, cudaEventDisableTiming);
        if (!e) e = cudaEventCreateWithFlags(&ctx->join_ev, cudaEventDisableTiming);
        if (e) return bail(fail(TITAN_ECUDA, std::string("closure stream: ") + cudaGetErrorString(e)));
    }
    for (auto& x : ctx->xev) {
        e = cudaEventCreateWithFlags(&x, cudaEventDisableTiming);
        if (e) return bail(fail(TITAN_ECUDA, std::string("cudaEventCreate: ") + cudaGetErrorString(e)));
    }

    e = cell_update_prepare();
    if (e) return bail(fail(TITAN_ECUDA, std::string("cell update kernels: ") + cudaGetErrorString(e)));

    // --- renumbering and remapped host arrays ---
    ctx->R = sfc_renumber(m->nnode, m->ncell, m->nface, m->node_xyz, m->cell_nodes, m->face_cells);
    const Renumbering& R = ctx->R;
    const int64_t nc = m->ncell, nf = m->nface, nn = m->nnode;
    std::vector<int32_t> face_c0(nf), face_c1(nf), face_bc(nf), face_nodes(4 * nf);
    std::vector<int8_t> face_type(nf), face_surf(nf), face_method(nf);
    for (int64_t f = 0; f < nf; ++f) {
        const int32_t o = R.face_n2o[f];
        face_c0[f] = R.cell_o2n[m->face_cells[2 * o]];
        const int32_t c1 = m->face_cells[2 * o + 1];
        face_c1[f] = c1 >= 0 ? R.cell_o2n[c1] : -1;
        face_type[f] = m->face_type[o];
        face_surf[f] = m->face_surf[o];
        face_method[f] = m->face_surf[o] != TITAN_SURF_US ? TITAN_HLLD : TITAN_LAX;  // Gran::Get_method
        face_bc[f] = m->face_bc[o];
        for (int k = 0; k < 4; ++k) face_nodes[k * nf + f] = R.node_o2n[m->face_nodes[4 * o + k]];
    }
    // The renumbering sorts faces by cells[0]: the first face owned by each
    // 32-cell chunk, for the staged cell update (empty if the order did not hold)
    std::vector<int32_t> owner_start;
    if (std::is_sorted(face_c0.begin(), face_c0.end())) {
        const int64_t nchunk = (nc + 31) / 32;
        owner_start.resize(nchunk + 1);
        int64_t f = 0;
        for (int64_t k = 0; k <= nchunk; ++k) {
            while (f < nf && face_c0[f] < 32 * k) ++f;
            owner_start[k] = (int32_t)f;
        }
    }
    std::vector<int32_t> cell_faces(6 * nc), cell_nodes(8 * nc);
    std::vector<int8_t> cell_type(nc);
    std::vector<uint8_t> cell_tvd(nc);
    for (int64_t c = 0; c < nc; ++c) {
        const int32_t o = R.cell_n2o[c];
        for (int s = 0; s < 6; ++s) {
            const int32_t fo = m->cell_faces[6 * o + s];
            int32_t fnew = R.face_o2n[fo];
            if (m->face_cells[2 * fo] != o) fnew |= (int32_t)0x80000000;  // sign -1 in the gather
            cell_faces[s * nc + c] = fnew;
        }
        for (int k = 0; k < 8; ++k) cell_nodes[k * nc + c] = R.node_o2n[m->cell_nodes[8 * o + k]];
        cell_type[c] = m->cell_type[o];
        cell_tvd[c] = m->cell_tvd[o];
    }
    // face slot -> the 4 face nodes as indices into the cell's 8 nodes (ALE geometry)
    std::vector<uint16_t> fmap;
    if (p->move) {
        fmap.resize(6 * nc);
        for (int64_t c = 0; c < nc; ++c) {
            const int64_t o = R.cell_n2o[c];
            for (int s = 0; s < 6; ++s) {
                const int32_t fo = m->cell_faces[6 * o + s];
                uint16_t code = 0;
                for (int k = 0; k < 4; ++k) {
                    int li = -1;
                    for (int j = 0; j < 8; ++j)
                        if (m->cell_nodes[8 * o + j] == m->face_nodes[4 * (int64_t)fo + k]) li = j;
                    if (li < 0) {
                        char buf[160];
                        snprintf(buf, sizeof buf, "face %d of cell %lld has a node the cell does not list", fo,
                                 (long long)o);
                        return bail(fail(TITAN_EMESH, buf));
                    }
                    code |= (uint16_t)(li << (3 * k));
                }
                fmap[s * nc + c] = code;
            }
        }
    }
    std::vector<double> xyz(3 * nn), amp, phase;
    for (int64_t i = 0; i < nn; ++i) {
        const int32_t o = R.node_n2o[i];
        for (int k = 0; k < 3; ++k) xyz[k * nn + i] = m->node_xyz[3 * o + k];
    }
    if (m->node_amp) {
        amp.resize(nn);
        phase.resize(nn);
        for (int64_t i = 0; i < nn; ++i) {
            amp[i] = m->node_amp[R.node_n2o[i]];
            phase[i] = m->node_phase[R.node_n2o[i]];
        }
    }
    std::vector<double> bc(TITAN_NV * std::max<int64_t>(m->nbc, 1), 0.0);
    for (int64_t r = 0; r < m->nbc; ++r)
        for (int k = 0; k < TITAN_NV; ++k) bc[k * m->nbc + r] = m->bc_vals[TITAN_NV * r + k];

    // --- device buffers ---
    int64_t& tot = ctx->dev_bytes;
#define DA(ptr, n)                                                                                     \
    do {                                                                                               \
        cudaError_t e_ = dalloc(&(ptr), (n), &tot);                                                    \
        if (e_) return bail(fail(TITAN_ENOMEM, std::string("cudaMalloc ") + #ptr + ": " + cudaGetErrorString(e_))); \
    } while (0)
    DA(ctx->d_cell_n2o, nc);
    DA(ctx->d_node_n2o, nn);
    DA(ctx->d_face_c0, nf);
    DA(ctx->d_face_c1, nf);
    DA(ctx->d_face_bc, nf);
    DA(ctx->d_face_nodes, 4 * nf);
    DA(ctx->d_face_type, nf);
    DA(ctx->d_face_surf, nf);
    DA(ctx->d_face_method, nf);
    DA(ctx->d_bc_vals, bc.size());
    DA(ctx->d_cell_faces, 6 * nc);
    if (!owner_start.empty()) DA(ctx->d_owner_start, owner_start.size());
    DA(ctx->d_cell_nodes, 8 * nc);
    DA(ctx->d_cell_type, nc);
    DA(ctx->d_cell_tvd, nc);
    if (m->node_amp) {
        DA(ctx->d_node_amp, nn);
        DA(ctx->d_node_phase, nn);
    }
    if (p->move) DA(ctx->d_cell_fmap, 6 * nc);
    if (p->tvd) {
        DA(ctx->d_face_aa, nf);
        DA(ctx->d_face_bb, nf);
    }
    const int nlayers = p->move ? 2 : 1;
    for (int l = 0; l < nlayers; ++l) {
        Layer& L = ctx->layer[l];
        DA(L.xyz, 3 * nn);
        DA(L.cc, 3 * nc);
        DA(L.vol, nc);
        DA(L.fc, 3 * nf);
        DA(L.fn, 3 * nf);
        DA(L.fa, nf);
        DA(L.fd, nf);
    }
    if (!p->move) ctx->layer[1] = ctx->layer[0];
    DA(ctx->d_state[0], (size_t)ctx->ns * nc);
    DA(ctx->d_state[1], (size_t)ctx->ns * nc);
    {
        const int n = 9 + p->npassive;
        ctx->flux_elem = 8;  // FP64 records in every mode
        ctx->flux_stride = (n + 1) & ~1;
        char* fp = nullptr;
        DA(fp, (size_t)nf * ctx->flux_stride * ctx->flux_elem);
        ctx->d_flux = fp;
    }
    if (p->nh > 0) DA(ctx->d_hfl, (size_t)5 * p->nh * nc);
    DA(ctx->d_stage, (size_t)TITAN_NV * std::max(nc, nn));
    DA(ctx->d_status, 1);
#undef DA
    e = cudaMallocHost((void**)&ctx->h_status, sizeof(DevStatus));
    if (e) return bail(fail(TITAN_ENOMEM, "cudaMallocHost status"));

    cudaStream_t s = ctx->stream;
    int rc = TITAN_OK;
    auto put = [&](auto* d, const auto& h) {
        if (rc) return;
        cudaError_t e_ = dput(d, h, s);
        if (e_) rc = fail(TITAN_ECUDA, cudaGetErrorString(e_));
    };
    put(ctx->d_cell_n2o, R.cell_n2o);
    put(ctx->d_node_n2o, R.node_n2o);
    put(ctx->d_face_c0, face_c0);
    put(ctx->d_face_c1, face_c1);
    put(ctx->d_face_bc, face_bc);
    put(ctx->d_face_nodes, face_nodes);
    put(ctx->d_face_type, face_type);
    put(ctx->d_face_surf, face_surf);
    put(ctx->d_face_method, face_method);
    put(ctx->d_bc_vals, bc);
    put(ctx->d_cell_faces, cell_faces);
    if (!owner_start.empty()) put(ctx->d_owner_start, owner_start);
    put(ctx->d_cell_nodes, cell_nodes);
    put(ctx->d_cell_type, cell_type);
    put(ctx->d_cell_tvd, cell_tvd);
    put(ctx->layer[0].xyz, xyz);
    if (m->node_amp) {
        put(ctx->d_node_amp, amp);
        put(ctx->d_node_phase, phase);
    }
    if (p->move) put(ctx->d_cell_fmap, fmap);
    if (rc) return bail(rc);
    e = cudaMemsetAsync(ctx->d_state[0], 0, sizeof(double) * ctx->ns * nc, s);
    if (!e) e = cudaMemsetAsync(ctx->d_state[1], 0, sizeof(double) * ctx->ns * nc, s);
    if (!e) e = cudaMemsetAsync(ctx->d_status, 0, sizeof(DevStatus), s);
    const MeshView M = ctx->view();
    if (!e) e = launch_cell_geometry(M, ctx->layer[0], s);
    if (!e) e = launch_face_geometry(M, ctx->layer[0], s);
    // second-order neighbours from the initial geometry (Setka::Init_TVD runs once, before Go)
    if (!e && p->tvd) e = launch_tvd_neighbours(M, ctx->layer[0], ctx->d_face_aa, ctx->d_face_bb, s);
    if (!e) e = cudaStreamSynchronize(s);
    if (e) return bail(fail(TITAN_ECUDA, std::string("create: ") + cudaGetErrorString(e)));
    *out = ctx;
    return TITAN_OK;
}

int titan_get_tvd_neighbours(titan_ctx* ctx, int32_t* out) {
    if (!ctx || !out) return fail(TITAN_EINVAL, "null argument");
    if (!ctx->P.tvd) return fail(TITAN_EINVAL, "context was created with tvd = 0");
    const int64_t nf = ctx->nface;
    std::vector<int32_t> aa(nf), bb(nf);
    CK(cudaMemcpyAsync(aa.data(), ctx->d_face_aa, sizeof(int32_t) * nf, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(bb.data(), ctx->d_face_bb, sizeof(int32_t) * nf, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    for (int64_t f = 0; f < nf; ++f) {
        const int64_t o = ctx->R.face_n2o[f];
        out[2 * o] = aa[f] >= 0 ? ctx->R.cell_n2o[aa[f]] : -1;
        out[2 * o + 1] = bb[f] >= 0 ? ctx->R.cell_n2o[bb[f]] : -1;
    }
    return TITAN_OK;
}

int titan_set_face_method(titan_ctx* ctx, const int8_t* ns) {
    if (!ctx || !ns) return fail(TITAN_EINVAL, "null argument");
    std::vector<int8_t> h(ctx->nface);
    for (int64_t f = 0; f < ctx->nface; ++f) {
        const int8_t v = ns[ctx->R.face_n2o[f]];
        if (v < 0 || v > 3) return fail(TITAN_EINVAL, "n_state must be 0..3");
        h[f] = v;
    }
    CK(cudaMemcpyAsync(ctx->d_face_method, h.data(), h.size(), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return TITAN_OK;
}

int titan_set_halo(titan_ctx* ctx, int64_t n_send, const int32_t* send_ids, int64_t n_recv,
                   const int32_t* recv_ids) {
    if (!ctx || n_send < 0 || n_recv < 0 || (n_send && !send_ids) || (n_recv && !recv_ids))
        return fail(TITAN_EINVAL, "bad argument");
    const int64_t nc = ctx->ncell;
    std::vector<int32_t> s(n_send), r(n_recv);
    for (int64_t i = 0; i < n_send; ++i) {
        if (send_ids[i] < 0 || send_ids[i] >= nc) return fail(TITAN_EINVAL, "halo cell id out of range");
        s[i] = ctx->R.cell_o2n[send_ids[i]];
    }
    for (int64_t i = 0; i < n_recv; ++i) {
        if (recv_ids[i] < 0 || recv_ids[i] >= nc) return fail(TITAN_EINVAL, "halo cell id out of range");
        r[i] = ctx->R.cell_o2n[recv_ids[i]];
    }
    if (ctx->d_halo_send) cudaFree(ctx->d_halo_send);
    if (ctx->d_halo_recv) cudaFree(ctx->d_halo_recv);
    ctx->d_halo_send = ctx->d_halo_recv = nullptr;
    ctx->n_halo_send = ctx->n_halo_recv = 0;
    int64_t tmp = 0;
    if (n_send) {
        CK(dalloc(&ctx->d_halo_send, (size_t)n_send, &tmp));
        CK(cudaMemcpy(ctx->d_halo_send, s.data(), sizeof(int32_t) * n_send, cudaMemcpyHostToDevice));
    }
    if (n_recv) {
        CK(dalloc(&ctx->d_halo_recv, (size_t)n_recv, &tmp));
        CK(cudaMemcpy(ctx->d_halo_recv, r.data(), sizeof(int32_t) * n_recv, cudaMemcpyHostToDevice));
    }
    ctx->n_halo_send = n_send;
    ctx->n_halo_recv = n_recv;
    return TITAN_OK;
}

int titan_set_cfl_faces(titan_ctx* ctx, const int8_t* exclude) {
    if (!ctx) return fail(TITAN_EINVAL, "null argument");
    drop_graph(ctx);  // the captured step reads the table's address
    if (ctx->d_face_nodt) cudaFree(ctx->d_face_nodt);
    ctx->d_face_nodt = nullptr;
    if (!exclude) return TITAN_OK;
    const int64_t nf = ctx->nface;
    std::vector<signed char> h(nf);
    for (int64_t f = 0; f < nf; ++f) h[f] = exclude[ctx->R.face_n2o[f]] ? 1 : 0;
    int64_t tmp = 0;
    CK(dalloc(&ctx->d_face_nodt, (size_t)nf, &tmp));
    CK(cudaMemcpy(ctx->d_face_nodt, h.data(), nf, cudaMemcpyHostToDevice));
    return TITAN_OK;
}

int titan_pack_halo(titan_ctx* ctx, double* out) {
    if (!ctx || (ctx->n_halo_send && !out)) return fail(TITAN_EINVAL, "bad argument");
    CK(launch_halo_pack(ctx->d_state[ctx->scur], (int)ctx->ncell, ctx->d_halo_send, (int)ctx->n_halo_send, ctx->ns,
                        out, ctx->stream));
    return TITAN_OK;
}

int titan_unpack_halo(titan_ctx* ctx, const double* in) {
    if (!ctx || (ctx->n_halo_recv && !in)) return fail(TITAN_EINVAL, "bad argument");
    CK(launch_halo_unpack(ctx->d_state[ctx->scur], (int)ctx->ncell, ctx->d_halo_recv, (int)ctx->n_halo_recv,
                          ctx->ns, in, ctx->stream));
    ctx->cl_valid = false;
    return TITAN_OK;
}

int titan_upload_state(titan_ctx* ctx, const double* state) {
    if (!ctx || !state) return fail(TITAN_EINVAL, "null argument");
    ctx->cl_valid = false;
    const int64_t nc = ctx->ncell;
    cudaStream_t s = ctx->stream, x = ctx->xfer;
    // field by field: the copy of field k+1 overlaps the gather of field k
    CK(cudaEventRecord(ctx->xev[TITAN_NV], s));  // earlier users of the staging buffer
    CK(cudaStreamWaitEvent(x, ctx->xev[TITAN_NV], 0));
    for (int k = 0; k < ctx->ns; ++k) {
        CK(cudaMemcpyAsync(ctx->d_stage + k * nc, state + k * nc, sizeof(double) * nc, cudaMemcpyHostToDevice, x));
        CK(cudaEventRecord(ctx->xev[k], x));
        CK(cudaStreamWaitEvent(s, ctx->xev[k], 0));
        CK(launch_gather(ctx->d_stage + k * nc, ctx->d_state[ctx->scur] + k * nc, ctx->d_cell_n2o, (int)nc, 1, s));
    }
    CK(cudaStreamSynchronize(s));
    return TITAN_OK;
}

int titan_download_state(titan_ctx* ctx, double* state) {
    if (!ctx || !state) return fail(TITAN_EINVAL, "null argument");
    const int64_t nc = ctx->ncell;
    cudaStream_t s = ctx->stream, x = ctx->xfer;
    // field by field: the copy of field k overlaps the scatter of field k+1
    for (int k = 0; k < ctx->ns; ++k) {
        CK(launch_scatter(ctx->d_state[ctx->scur] + k * nc, ctx->d_stage + k * nc, ctx->d_cell_n2o, (int)nc, 1, s));
        CK(cudaEventRecord(ctx->xev[k], s));
    }
    for (int k = 0; k < ctx->ns; ++k) {
        CK(cudaStreamWaitEvent(x, ctx->xev[k], 0));
        CK(cudaMemcpyAsync(state + k * nc, ctx->d_stage + k * nc, sizeof(double) * nc, cudaMemcpyDeviceToHost, x));
    }
    CK(cudaStreamSynchronize(x));
    return TITAN_OK;
}

int titan_upload_hfluids(titan_ctx* ctx, const double* h) {
    if (!ctx || !h) return fail(TITAN_EINVAL, "null argument");
    if (ctx->prm.nh <= 0) return fail(TITAN_EINVAL, "context was created with nh = 0");
    const int64_t nc = ctx->ncell;
    const int nfields = 5 * ctx->prm.nh;
    for (int k0 = 0; k0 < nfields; k0 += TITAN_NV) {
        const int nk = std::min(TITAN_NV, nfields - k0);
        CK(cudaMemcpyAsync(ctx->d_stage, h + (size_t)k0 * nc, sizeof(double) * nk * nc, cudaMemcpyHostToDevice,
                           ctx->stream));
        CK(launch_gather(ctx->d_stage, ctx->d_hfl + (size_t)k0 * nc, ctx->d_cell_n2o, (int)nc, nk, ctx->stream));
    }
    CK(cudaStreamSynchronize(ctx->stream));
    return TITAN_OK;
}

int titan_set_sources(titan_ctx* ctx, const double* src) {
    if (!ctx) return fail(TITAN_EINVAL, "null argument");
    drop_graph(ctx);
    if (!src) {
        ctx->use_src = false;
        return TITAN_OK;
    }
    const int64_t nc = ctx->ncell;
    if (!ctx->d_src) {
        int64_t dummy = 0;
        CK(dalloc(&ctx->d_src, (size_t)4 * nc, &dummy));
        ctx->dev_bytes += dummy;
    }
    CK(cudaMemcpyAsync(ctx->d_stage, src, sizeof(double) * 4 * nc, cudaMemcpyHostToDevice, ctx->stream));
    CK(launch_gather(ctx->d_stage, ctx->d_src, ctx->d_cell_n2o, (int)nc, 4, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->use_src = true;
    return TITAN_OK;
}

}  // extern "C"

namespace {

// The device clock and status word of a run: dt, t, cleared counters and error
// word, the identity of the CFL minimum; written by a kernel, so it is
// ordered on the stream like the steps and needs no host buffer.
__global__ void set_status_kernel(DevStatus* st, double dt, double t) {
    st->err_kind = 0;
    st->err_index = 0;
    st->n_rho_floor = 0;
    st->n_p_floor = 0;
    st->steps_done = 0;
    st->block_counter = 0;
    st->dt_next_bits = 0x4197D78400000000ull;  // bits of 1e8, the identity of the CFL minimum
    st->dt = dt;
    st->t = t;
}

// Enqueues nsteps steps on the context's stream from the device clock; no host sync.
int enqueue_steps(titan_ctx* ctx, int64_t nsteps) {
    cudaStream_t s = ctx->stream;
    if (ctx->use_closure && !ctx->cl_valid && nsteps > 0) {
        // the state or centres changed outside the step loop: the closure's
        // inputs for the first step (every later step's come from the cell update)
        CK(timed(ctx, "closure_inputs", [&] {
            return launch_closure_inputs(ctx->d_state[ctx->scur], ctx->layer[ctx->cur].cc, (int)ctx->ncell,
                                         ctx->closure.norm, ctx->d_env, ctx->closure_ninf, ctx->closure_lambda,
                                         ctx->d_cl_in, ctx->d_cl_out, s);
        }));
        ctx->cl_valid = true;
    }
    int64_t done = 0;
    if (ctx->profiling) {
        drop_graph(ctx);
        for (; done < nsteps; ++done) CK(enqueue_step(ctx));
    } else {
        // The graph holds two steps; its pointers are fixed for one buffer phase.
        if (nsteps >= 2 && (ctx->graph == nullptr || ctx->graph_cur != ctx->cur || ctx->graph_scur != ctx->scur))
            CK(capture_two_steps(ctx));
        for (; done + 2 <= nsteps; done += 2) CK(cudaGraphLaunch(ctx->graph, s));
        for (; done < nsteps; ++done) {
            // The graph's two-step period leaves the buffers in the captured
            // phase; a final odd step runs eagerly.
            CK(enqueue_step(ctx));
        }
    }
    return TITAN_OK;
}

// Waits for the context's stream and reports the device clock and status.
int finish_steps(titan_ctx* ctx, double* dt_out, double* t_out, titan_step_info* info, float ms) {
    cudaStream_t s = ctx->stream;
    CK(cudaMemcpyAsync(ctx->h_status, ctx->d_status, sizeof(DevStatus), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    const DevStatus& st = *ctx->h_status;
    if (dt_out) *dt_out = st.dt;
    if (t_out) *t_out = st.t;
    int status = TITAN_OK;
    if (st.err_kind != 0)
        status = st.err_kind == 21 ? TITAN_ETIMEOUT : st.err_kind >= 20 ? TITAN_ENONFINITE : TITAN_ESOLVER;
    if (ctx->use_closure) {
        int cerr = 0;
        CK(cudaMemcpy(&cerr, ctx->closure.error, sizeof(int), cudaMemcpyDeviceToHost));
        if (cerr) return fail(TITAN_ETIMEOUT, "closure: a tensor-core wait ran out");
    }
    if (info) {
        info->steps_done = (int64_t)st.steps_done;
        info->n_rho_floor = (int64_t)st.n_rho_floor;
        info->n_p_floor = (int64_t)st.n_p_floor;
        info->status = status;
        info->err_kind = st.err_kind;
        info->err_index = -1;
        if (st.err_kind != 0) {
            const int idx = st.err_index;
            if (st.err_kind >= 20)  // a cell (20) or the first cell of a block (21)
                info->err_index = (idx >= 0 && idx < ctx->ncell) ? ctx->R.cell_n2o[idx] : -1;
            else
                info->err_index = (idx >= 0 && idx < ctx->nface) ? ctx->R.face_n2o[idx] : -1;
        }
        info->dt_next = st.dt;
        info->t = st.t;
        info->gpu_ms = ms;
    }
    if (status != TITAN_OK) {
        char buf[160];
        snprintf(buf, sizeof buf, "step failed: kind %d at renumbered index %d after %llu steps", st.err_kind,
                 st.err_index, (unsigned long long)st.steps_done);
        return fail(status, buf);
    }
    return TITAN_OK;
}

}  // namespace

extern "C" {

int titan_step(titan_ctx* ctx, int64_t nsteps, double* dt_inout, double* t_inout, titan_step_info* info) {
    if (!ctx || !dt_inout || nsteps < 0) return fail(TITAN_EINVAL, "bad argument");
    const double t0 = t_inout ? *t_inout : 0.0;
    if (!(*dt_inout > 0.0) || !std::isfinite(*dt_inout)) return fail(TITAN_EINVAL, "dt must be positive");
    cudaStream_t s = ctx->stream;
    set_status_kernel<<<1, 1, 0, s>>>(ctx->d_status, *dt_inout, t0);
    CK(cudaGetLastError());
    CK(cudaEventRecord(ctx->ev[0], s));
    const int rc = enqueue_steps(ctx, nsteps);
    if (rc) return rc;
    CK(cudaEventRecord(ctx->ev[1], s));
    CK(cudaEventSynchronize(ctx->ev[1]));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
    return finish_steps(ctx, dt_inout, t_inout, info, ms);
}

int titan_set_clock(titan_ctx* ctx, double dt, double t) {
    if (!ctx) return fail(TITAN_EINVAL, "null argument");
    if (!(dt > 0.0) || !std::isfinite(dt) || !std::isfinite(t)) return fail(TITAN_EINVAL, "dt must be positive");
    set_status_kernel<<<1, 1, 0, ctx->stream>>>(ctx->d_status, dt, t);
    CK(cudaGetLastError());
    return TITAN_OK;
}

int titan_step_async(titan_ctx* ctx, int64_t nsteps) {
    if (!ctx || nsteps < 0) return fail(TITAN_EINVAL, "bad argument");
    return enqueue_steps(ctx, nsteps);
}

int titan_get_clock(titan_ctx* ctx, double* dt, double* t, titan_step_info* info) {
    if (!ctx) return fail(TITAN_EINVAL, "null argument");
    return finish_steps(ctx, dt, t, info, 0.f);
}

int titan_dt_copy(titan_ctx* ctx, double* dev, int32_t into_clock) {
    if (!ctx || !dev) return fail(TITAN_EINVAL, "null argument");
    double* clock_dt = &ctx->d_status->dt;
    CK(cudaMemcpyAsync(into_clock ? clock_dt : dev, into_clock ? dev : clock_dt, sizeof(double),
                       cudaMemcpyDeviceToDevice, ctx->stream));
    return TITAN_OK;
}

int titan_upload_nodes(titan_ctx* ctx, const double* xyz) {
    if (!ctx || !xyz) return fail(TITAN_EINVAL, "null argument");
    const int64_t nn = ctx->nnode;
    for (int64_t i = 0; i < 3 * nn; ++i)
        if (!std::isfinite(xyz[i])) return fail(TITAN_EINVAL, "non-finite node coordinate");
    std::vector<double> h(3 * nn);
    for (int64_t i = 0; i < nn; ++i)
        for (int k = 0; k < 3; ++k) h[k * nn + i] = xyz[3 * (int64_t)ctx->R.node_n2o[i] + k];
    drop_graph(ctx);
    ctx->cl_valid = false;
    const Layer& L = ctx->layer[ctx->cur];
    CK(cudaMemcpyAsync(L.xyz, h.data(), sizeof(double) * 3 * nn, cudaMemcpyHostToDevice, ctx->stream));
    const MeshView M = ctx->view();
    CK(launch_cell_geometry(M, L, ctx->stream));
    CK(launch_face_geometry(M, L, ctx->stream));
    // as in the reference, where Init_TVD runs after Download_cell_parameters
    if (ctx->P.tvd) CK(launch_tvd_neighbours(M, L, ctx->d_face_aa, ctx->d_face_bb, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return TITAN_OK;
}

int titan_download_nodes(titan_ctx* ctx, double* xyz) {
    if (!ctx || !xyz) return fail(TITAN_EINVAL, "null argument");
    const int64_t nn = ctx->nnode;
    std::vector<double> h(3 * nn);
    CK(cudaMemcpyAsync(h.data(), ctx->layer[ctx->cur].xyz, sizeof(double) * 3 * nn, cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    for (int64_t i = 0; i < nn; ++i)
        for (int k = 0; k < 3; ++k) xyz[3 * (int64_t)ctx->R.node_n2o[i] + k] = h[k * nn + i];
    return TITAN_OK;
}

int titan_download_geometry(titan_ctx* ctx, double* cc, double* vol, double* fc, double* fn, double* fa) {
    if (!ctx) return fail(TITAN_EINVAL, "null argument");
    const int64_t nc = ctx->ncell, nf = ctx->nface;
    const Layer& L = ctx->layer[ctx->cur];
    // a moving mesh keeps only node and cell geometry between steps
    if (ctx->prm.move) CK(launch_face_geometry(ctx->view(), L, ctx->stream));
    std::vector<double> hcc(3 * nc), hvol(nc), hfc(3 * nf), hfn(3 * nf), hfa(nf);
    CK(cudaMemcpyAsync(hcc.data(), L.cc, sizeof(double) * 3 * nc, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(hvol.data(), L.vol, sizeof(double) * nc, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(hfc.data(), L.fc, sizeof(double) * 3 * nf, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(hfn.data(), L.fn, sizeof(double) * 3 * nf, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(hfa.data(), L.fa, sizeof(double) * nf, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    for (int64_t c = 0; c < nc; ++c) {
        const int64_t o = ctx->R.cell_n2o[c];
        if (cc)
            for (int k = 0; k < 3; ++k) cc[3 * o + k] = hcc[k * nc + c];
        if (vol) vol[o] = hvol[c];
    }
    for (int64_t f = 0; f < nf; ++f) {
        const int64_t o = ctx->R.face_n2o[f];
        for (int k = 0; k < 3; ++k) {
            if (fc) fc[3 * o + k] = hfc[k * nf + f];
            if (fn) fn[3 * o + k] = hfn[k * nf + f];
        }
        if (fa) fa[o] = hfa[f];
    }
    return TITAN_OK;
}

int titan_download_face_fluxes(titan_ctx* ctx, double* flux) {
    if (!ctx || !flux) return fail(TITAN_EINVAL, "null argument");
    const int64_t nf = ctx->nface;
    const int stride = ctx->flux_stride;
    std::vector<char> raw((size_t)nf * stride * ctx->flux_elem);
    CK(cudaMemcpyAsync(raw.data(), ctx->d_flux, raw.size(), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    const int n = 9 + ctx->prm.npassive;
    for (int64_t f = 0; f < nf; ++f) {
        double* dst = flux + 11 * (int64_t)ctx->R.face_n2o[f];
        for (int k = 0; k < 11; ++k) {
            double v = 0.0;
            if (k < n) v = reinterpret_cast<const double*>(raw.data())[(size_t)f * stride + k];
            dst[k] = v;
        }
    }
    return TITAN_OK;
}

int titan_sfc_renumber(int64_t nnode, int64_t ncell, int64_t nface, const double* xyz, const int32_t* cell_nodes,
                       const int32_t* face_cells, int32_t* cells, int32_t* faces, int32_t* nodes) {
    if (nnode <= 0 || ncell <= 0 || nface <= 0 || !xyz || !cell_nodes || !face_cells)
        return fail(TITAN_EINVAL, "bad argument");
    for (int64_t i = 0; i < 8 * ncell; ++i)
        if (cell_nodes[i] < 0 || cell_nodes[i] >= nnode) return fail(TITAN_EMESH, "cell node index out of range");
    for (int64_t f = 0; f < nface; ++f)
        if (face_cells[2 * f] < 0 || face_cells[2 * f] >= ncell) return fail(TITAN_EMESH, "cells[0] out of range");
    const Renumbering R = sfc_renumber(nnode, ncell, nface, xyz, cell_nodes, face_cells);
    if (cells) std::memcpy(cells, R.cell_n2o.data(), sizeof(int32_t) * ncell);
    if (faces) std::memcpy(faces, R.face_n2o.data(), sizeof(int32_t) * nface);
    if (nodes) std::memcpy(nodes, R.node_n2o.data(), sizeof(int32_t) * nnode);
    return TITAN_OK;
}

int titan_get_permutation(titan_ctx* ctx, int32_t* cells, int32_t* faces, int32_t* nodes) {
    if (!ctx) return fail(TITAN_EINVAL, "null argument");
    if (cells) std::memcpy(cells, ctx->R.cell_n2o.data(), sizeof(int32_t) * ctx->ncell);
    if (faces) std::memcpy(faces, ctx->R.face_n2o.data(), sizeof(int32_t) * ctx->nface);
    if (nodes) std::memcpy(nodes, ctx->R.node_n2o.data(), sizeof(int32_t) * ctx->nnode);
    return TITAN_OK;
}

int titan_riemann_batch(int64_t n, const int8_t* n_state, const double* nrm, const double* w, const double* q1,
                        const double* q2, int32_t flags, int32_t precision, double gamma, double* flux,
                        double* ds, int32_t* rc) {
    if (n < 0 || (n > 0 && (!n_state || !nrm || !w || !q1 || !q2 || !flux || !ds || !rc)))
        return fail(TITAN_EINVAL, "bad argument");
    if (precision != 64 && precision != 32) return fail(TITAN_EINVAL, "precision must be 64 or 32");
    if (n == 0) return TITAN_OK;
    signed char* dns = nullptr;
    double *dn = nullptr, *dw = nullptr, *d1 = nullptr, *d2 = nullptr, *df = nullptr, *dd = nullptr;
    int* drc = nullptr;
    int64_t tot = 0;
    cudaError_t e = cudaSuccess;
    if (!e) e = dalloc(&dns, n, &tot);
    if (!e) e = dalloc(&dn, 3 * n, &tot);
    if (!e) e = dalloc(&dw, n, &tot);
    if (!e) e = dalloc(&d1, 8 * n, &tot);
    if (!e) e = dalloc(&d2, 8 * n, &tot);
    if (!e) e = dalloc(&df, 8 * n, &tot);
    if (!e) e = dalloc(&dd, 3 * n, &tot);
    if (!e) e = dalloc(&drc, n, &tot);
    if (!e) e = cudaMemcpy(dns, n_state, n, cudaMemcpyHostToDevice);
    if (!e) e = cudaMemcpy(dn, nrm, sizeof(double) * 3 * n, cudaMemcpyHostToDevice);
    if (!e) e = cudaMemcpy(dw, w, sizeof(double) * n, cudaMemcpyHostToDevice);
    if (!e) e = cudaMemcpy(d1, q1, sizeof(double) * 8 * n, cudaMemcpyHostToDevice);
    if (!e) e = cudaMemcpy(d2, q2, sizeof(double) * 8 * n, cudaMemcpyHostToDevice);
    if (!e)
        e = precision == 64 ? launch_riemann_batch_fp64(n, dns, dn, dw, d1, d2, df, dd, drc, flags, gamma, 0)
                            : launch_riemann_batch_fp32(n, dns, dn, dw, d1, d2, df, dd, drc, flags, gamma, 0);
    if (!e) e = cudaMemcpy(flux, df, sizeof(double) * 8 * n, cudaMemcpyDeviceToHost);
    if (!e) e = cudaMemcpy(ds, dd, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost);
    if (!e) e = cudaMemcpy(rc, drc, sizeof(int) * n, cudaMemcpyDeviceToHost);
    void* ps[] = {dns, dn, dw, d1, d2, df, dd, drc};
    for (void* p : ps)
        if (p) cudaFree(p);
    if (e) return fail(TITAN_ECUDA, std::string("riemann_batch: ") + cudaGetErrorString(e));
    return TITAN_OK;
}

int titan_set_closure(titan_ctx* ctx, const float* params, const float* norm, double n_inf, double lambda) {
    if (!ctx) return fail(TITAN_EINVAL, "null argument");
    drop_graph(ctx);
    closure_destroy(&ctx->closure);
    ctx->use_closure = false;
    if (!params) return TITAN_OK;
    if (!norm || !(n_inf > 0.0)) return fail(TITAN_EINVAL, "closure needs norm and n_inf > 0");
    if (!ctx->d_cl_in) {
        int64_t bytes = 0;
        cudaError_t e = dalloc(&ctx->d_cl_in, (size_t)8 * ctx->ncell, &bytes);
        if (!e) e = dalloc(&ctx->d_cl_y, (size_t)5 * ctx->ncell, &bytes);
        if (!e) e = dalloc(&ctx->d_cl_out, (size_t)ctx->ncell, &bytes);
        if (e) return fail(TITAN_ENOMEM, std::string("closure buffers: ") + cudaGetErrorString(e));
        ctx->dev_bytes += bytes;
    }
    ctx->cl_valid = false;
    int dev = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, dev));
    cudaError_t e = closure_create(params, norm, &ctx->closure, ctx->stream);
    if (e) {
        closure_destroy(&ctx->closure);
        return fail(TITAN_ECUDA, std::string("closure: ") + cudaGetErrorString(e));
    }
    ctx->closure_ninf = n_inf;
    ctx->closure_lambda = lambda;
    ctx->use_closure = true;
    return TITAN_OK;
}

int titan_godunov_batch(int64_t n, const double* nrm, const double* w, const double* q1, const double* q2,
                        const int8_t* contact, double gamma, double* flux, double* ds, int32_t* rc) {
    if (n <= 0 || !nrm || !w || !q1 || !q2 || !contact || !flux || !ds || !rc)
        return fail(TITAN_EINVAL, "titan_godunov_batch: bad argument");
    double *dn = nullptr, *dw = nullptr, *d1 = nullptr, *d2 = nullptr, *df = nullptr, *dd = nullptr;
    int8_t* dc = nullptr;
    int* drc = nullptr;
    auto release = [&] {
        void* ps[] = {dn, dw, d1, d2, df, dd, dc, drc};
        for (void* p : ps)
            if (p) cudaFree(p);
    };
    cudaError_t e = cudaMalloc((void**)&dn, sizeof(double) * 3 * n);
    if (!e) e = cudaMalloc((void**)&dw, sizeof(double) * n);
    if (!e) e = cudaMalloc((void**)&d1, sizeof(double) * 5 * n);
    if (!e) e = cudaMalloc((void**)&d2, sizeof(double) * 5 * n);
    if (!e) e = cudaMalloc((void**)&df, sizeof(double) * 5 * n);
    if (!e) e = cudaMalloc((void**)&dd, sizeof(double) * 3 * n);
    if (!e) e = cudaMalloc((void**)&dc, n);
    if (!e) e = cudaMalloc((void**)&drc, sizeof(int) * n);
    if (!e) e = cudaMemcpy(dn, nrm, sizeof(double) * 3 * n, cudaMemcpyHostToDevice);
    if (!e) e = cudaMemcpy(dw, w, sizeof(double) * n, cudaMemcpyHostToDevice);
    if (!e) e = cudaMemcpy(d1, q1, sizeof(double) * 5 * n, cudaMemcpyHostToDevice);
    if (!e) e = cudaMemcpy(d2, q2, sizeof(double) * 5 * n, cudaMemcpyHostToDevice);
    if (!e) e = cudaMemcpy(dc, contact, n, cudaMemcpyHostToDevice);
    if (!e) e = launch_godunov_batch(n, dn, dw, d1, d2, reinterpret_cast<const signed char*>(dc), gamma, df, dd, drc, 0);
    if (!e) e = cudaMemcpy(flux, df, sizeof(double) * 5 * n, cudaMemcpyDeviceToHost);
    if (!e) e = cudaMemcpy(ds, dd, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost);
    if (!e) e = cudaMemcpy(rc, drc, sizeof(int) * n, cudaMemcpyDeviceToHost);
    release();
    if (e) return fail(TITAN_ECUDA, std::string("titan_godunov_batch: ") + cudaGetErrorString(e));
    return TITAN_OK;
}

int titan_set_closure_fallback(titan_ctx* ctx, const float* lo, const float* hi, const double* src) {
    if (!ctx) return fail(TITAN_EINVAL, "null argument");
    if ((lo == nullptr) != (hi == nullptr)) return fail(TITAN_EINVAL, "lo and hi go together");
    drop_graph(ctx);
    ctx->cl_valid = false;  // the envelope flags are formed with the inputs
    if (!lo) {
        void* ps[] = {ctx->d_env, ctx->d_fallback, ctx->d_n_outside};
        for (void* p : ps)
            if (p) cudaFree(p);
        ctx->d_env = nullptr;
        ctx->d_fallback = nullptr;
        ctx->d_n_outside = nullptr;
        return TITAN_OK;
    }
    const int64_t nc = ctx->ncell;
    int64_t dummy = 0;
    if (!ctx->d_env) CK(dalloc(&ctx->d_env, 2 * kIn, &dummy));
    if (!ctx->d_n_outside) {
        CK(dalloc(&ctx->d_n_outside, 1, &dummy));
        CK(cudaMemsetAsync(ctx->d_n_outside, 0, sizeof(unsigned long long), ctx->stream));
    }
    float env[2 * kIn];
    for (int k = 0; k < kIn; ++k) {
        env[k] = lo[k];
        env[kIn + k] = hi[k];
    }
    CK(cudaMemcpyAsync(ctx->d_env, env, sizeof(env), cudaMemcpyHostToDevice, ctx->stream));
    if (src) {
        if (!ctx->d_fallback) CK(dalloc(&ctx->d_fallback, (size_t)4 * nc, &dummy));
        CK(cudaMemcpyAsync(ctx->d_stage, src, sizeof(double) * 4 * nc, cudaMemcpyHostToDevice, ctx->stream));
        CK(launch_gather(ctx->d_stage, ctx->d_fallback, ctx->d_cell_n2o, (int)nc, 4, ctx->stream));
    }
    CK(cudaStreamSynchronize(ctx->stream));
    return TITAN_OK;
}

int titan_closure_fallback_from_mc(titan_ctx* ctx) {
    if (!ctx) return fail(TITAN_EINVAL, "null argument");
    if (!ctx->d_env) return fail(TITAN_EINVAL, "no closure envelope: call titan_set_closure_fallback first");
    if (!ctx->mc_valid) return fail(TITAN_EINVAL, "no Monte-Carlo pass on this context");
    const int64_t nc = ctx->ncell;
    if (!ctx->d_fallback) {
        int64_t dummy = 0;
        CK(dalloc(&ctx->d_fallback, (size_t)4 * nc, &dummy));
        drop_graph(ctx);  // the captured step reads the table's address
    }
    // the tallies are in the device's cell numbering, as the table is
    CK(cudaMemcpyAsync(ctx->d_fallback, ctx->d_mc_tally + nc, sizeof(double) * 4 * nc, cudaMemcpyDeviceToDevice,
                       ctx->stream));
    return TITAN_OK;
}

int titan_closure_outside(titan_ctx* ctx, int64_t* n_outside) {
    if (!ctx || !n_outside) return fail(TITAN_EINVAL, "null argument");
    unsigned long long v = 0;
    if (ctx->d_n_outside)
        CK(cudaMemcpy(&v, ctx->d_n_outside, sizeof(v), cudaMemcpyDeviceToHost));
    *n_outside = (int64_t)v;
    return TITAN_OK;
}

int titan_mc_sources(titan_ctx* ctx, const titan_mc_params* mp, double* out, titan_mc_info* info) {
    if (!ctx || !mp) return fail(TITAN_EINVAL, "null argument");
    if (mp->n_particles <= 0 || !(mp->n_H > 0.0) || !(mp->cp_H > 0.0)) return fail(TITAN_EINVAL, "bad MC parameters");
    const int64_t nc = ctx->ncell, nf = ctx->nface;
    cudaStream_t s = ctx->stream;
    const MeshView M = ctx->view();
    const Layer& L = ctx->layer[ctx->cur];
    if (ctx->prm.move) CK(launch_face_geometry(M, L, s));  // faces of the current layer
    const int nb = mc_scan_blocks(nf);
    if (!ctx->d_mc_cells) {
        int64_t tmp = 0;
        cudaError_t e = dalloc(&ctx->d_mc_cells, (size_t)nc, &tmp);
        if (!e) e = dalloc(&ctx->d_mc_cdf, (size_t)nf, &tmp);
        if (!e) e = dalloc(&ctx->d_mc_blocks, (size_t)nb + 1, &tmp);
        if (!e) e = dalloc(&ctx->d_mc_tally, (size_t)5 * nc, &tmp);
        if (!e) e = dalloc(&ctx->d_mc_lost, 1, &tmp);
        if (e) {
            void* ps[] = {ctx->d_mc_cells, ctx->d_mc_cdf, ctx->d_mc_blocks, ctx->d_mc_tally, ctx->d_mc_lost};
            for (void* p : ps)
                if (p) cudaFree(p);
            ctx->d_mc_cells = nullptr;
            ctx->d_mc_cdf = ctx->d_mc_blocks = ctx->d_mc_tally = nullptr;
            ctx->d_mc_lost = nullptr;
            return fail(TITAN_ECUDA, std::string("mc buffers: ") + cudaGetErrorString(e));
        }
    }
    ctx->mc_valid = false;
    double* d_total = ctx->d_mc_blocks + nb;
    McArgs a{};
    a.M = M;
    a.P = ctx->P;
    a.L = L;
    a.state = ctx->d_state[ctx->scur];
    a.inflow_cdf = ctx->d_mc_cdf;
    a.nparticles = mp->n_particles;
    a.nH = mp->n_H;
    a.uH0 = mp->u_H[0];
    a.uH1 = mp->u_H[1];
    a.uH2 = mp->u_H[2];
    a.cpH = mp->cp_H;
    a.face_types = (unsigned)mp->face_types;
    a.seed = mp->seed;
    a.max_cells = mp->max_cells > 0 ? mp->max_cells : 1000000;
    a.tally = ctx->d_mc_tally;
    a.lost = ctx->d_mc_lost;
    if (ctx->fd_buf[0]) {
        a.fd.index = (const int*)ctx->fd_buf[0];
        a.fd.frame = (const double*)ctx->fd_buf[1];
        a.fd.side = (const signed char*)ctx->fd_buf[2];
        a.fd.flux = (const double*)ctx->fd_buf[3];
        a.fd.leaf_ptr = (const int*)ctx->fd_buf[4];
        a.fd.box = (const double*)ctx->fd_buf[5];
        a.fd.cum = (const double*)ctx->fd_buf[6];
    }
    if (ctx->ft_buf[0]) {
        a.ft.index = (const int*)ctx->ft_buf[0];
        a.ft.face = (const int*)ctx->ft_buf[1];
        a.ft.side = (const signed char*)ctx->ft_buf[2];
        a.ft.frame = (const double*)ctx->ft_buf[3];
        a.ft.bounds = (const double*)ctx->ft_buf[4];
        a.ft.leaf_ptr = (const int*)ctx->ft_buf[5];
        a.ft.box = (const double*)ctx->ft_buf[6];
        a.ft.f = (double*)ctx->ft_buf[7];
        a.ft.mom = (double*)ctx->ft_buf[8];
        a.ft.unplaced = (unsigned long long*)ctx->ft_buf[9];
        ctx->ft_valid = false;
    }
    // per-neutral end records (tests and diagnostics): a buffer for this pass only
    struct TraceBuf {
        double* p = nullptr;
        ~TraceBuf() {
            if (p) cudaFree(p);
        }
    } trace;
    if (mp->trace_out) {
        int64_t tmp = 0;
        cudaError_t e = dalloc(&trace.p, (size_t)8 * (size_t)mp->n_particles, &tmp);
        if (e) return fail(TITAN_ENOMEM, std::string("mc trace buffer: ") + cudaGetErrorString(e));
        a.trace = trace.p;
    }
    // inflow CDF on the device; its total sets the particle weight
    double total = 0.0;
    CK(cudaEventRecord(ctx->ev[0], s));
    CK(launch_mc_inflow_cdf(a, ctx->d_mc_cdf, ctx->d_mc_blocks, d_total, s));
    CK(cudaMemcpyAsync(&total, d_total, sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (!(total > 0.0)) return fail(TITAN_EINVAL, "no inflow faces of the requested types");
    a.mu = total / (double)mp->n_particles;
    CK(cudaMemsetAsync(ctx->d_mc_tally, 0, sizeof(double) * 5 * nc, s));
    CK(cudaMemsetAsync(ctx->d_mc_lost, 0, sizeof(unsigned long long), s));
    if (a.ft.index) {
        CK(cudaMemsetAsync(a.ft.f, 0, sizeof(double) * ctx->ft_nleaf, s));
        CK(cudaMemsetAsync(a.ft.mom, 0, sizeof(double) * 3 * ctx->ft_ntab, s));
        CK(cudaMemsetAsync(a.ft.unplaced, 0, sizeof(unsigned long long), s));
    }
    CK(launch_mc_pack(a, ctx->d_mc_cells, s));
    CK(launch_mc_trace_cells(a, ctx->d_mc_cells, s));
    CK(launch_mc_normalise(ctx->d_mc_tally, L.vol, (int)nc, s));
    if (a.ft.index) CK(launch_mc_tally_normalise(a, (int)ctx->ft_ntab, s));
    // back to the caller's cell numbering on the device, then one copy
    if (out) CK(launch_scatter(ctx->d_mc_tally, ctx->d_stage, ctx->d_cell_n2o, (int)nc, 5, s));
    CK(cudaEventRecord(ctx->ev[1], s));
    unsigned long long lost = 0;
    if (out) CK(cudaMemcpyAsync(out, ctx->d_stage, sizeof(double) * 5 * nc, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(&lost, ctx->d_mc_lost, sizeof(lost), cudaMemcpyDeviceToHost, s));
    if (mp->trace_out)
        CK(cudaMemcpyAsync(mp->trace_out, trace.p, sizeof(double) * 8 * (size_t)mp->n_particles,
                           cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]));
    ctx->mc_valid = true;
    ctx->ft_valid = a.ft.index != nullptr;
    if (info) {
        info->particles = mp->n_particles;
        info->lost = (int64_t)lost;
        info->inflow_rate = total;
        info->gpu_ms = ms;
    }
    return TITAN_OK;
}

int titan_set_mc_face_dist(titan_ctx* ctx, const titan_mc_face_dist* d) {
    if (!ctx) return fail(TITAN_EINVAL, "null argument");
    for (void*& p : ctx->fd_buf) {
        if (p) cudaFree(p);
        p = nullptr;
    }
    if (!d || d->nface == 0) return TITAN_OK;
    if (d->nface < 0 || !d->face || !d->side || !d->frame || !d->leaf_ptr || !d->leaf_box || !d->leaf_f)
        return fail(TITAN_EINVAL, "face tables: nface >= 0 and every array");
    const int64_t nf = ctx->nface, nt = d->nface;
    const Renumbering& R = ctx->R;
    if (d->leaf_ptr[0] != 0) return fail(TITAN_EINVAL, "face tables: leaf_ptr[0] must be 0");
    const int64_t nleaf = d->leaf_ptr[nt];
    if (nleaf < nt || nleaf > INT32_MAX) return fail(TITAN_EINVAL, "face tables: leaf_ptr[nface] out of range");
    std::vector<int32_t> index(nf, -1), ptr(nt + 1, 0);
    std::vector<int8_t> side(nt);
    std::vector<double> flux(nt), cum(nleaf);
    std::vector<int32_t> c1(nf);
    CK(cudaMemcpy(c1.data(), ctx->d_face_c1, sizeof(int32_t) * nf, cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < nt; ++i) {
        const int32_t fo = d->face[i];
        if (fo < 0 || fo >= nf) return fail(TITAN_EINVAL, "face tables: face id out of range");
        const int32_t f = R.face_o2n[fo];
        if (index[f] >= 0) return fail(TITAN_EINVAL, "face tables: a face is listed twice");
        index[f] = (int32_t)i;
        if (d->side[i] != 0 && d->side[i] != 1) return fail(TITAN_EINVAL, "face tables: side is 0 or 1");
        if (d->side[i] == 1 && c1[f] < 0) return fail(TITAN_EINVAL, "face tables: side 1 on a boundary face");
        side[i] = d->side[i];
        const int64_t l0 = d->leaf_ptr[i], l1 = d->leaf_ptr[i + 1];
        if (!(l1 > l0) || l1 > nleaf) return fail(TITAN_EINVAL, "face tables: leaf_ptr must increase to leaf_ptr[nface]");
        ptr[i + 1] = (int32_t)l1;
        // inflow per unit area: leaf weights box volume * f * |centre x| summed
        // in the given (tree) order, then each leaf's cumulative share
        double sum = 0.0;
        for (int64_t l = l0; l < l1; ++l) {
            const double* b = d->leaf_box + 6 * l;
            const double fl = d->leaf_f[l];
            if (!(b[0] >= 0.0 && b[1] > b[0] && b[3] > b[2] && b[5] > b[4]) || !(fl >= 0.0) || !std::isfinite(fl) ||
                !std::isfinite(b[1]) || !std::isfinite(b[2]) || !std::isfinite(b[3]) || !std::isfinite(b[4]) ||
                !std::isfinite(b[5]))
                return fail(TITAN_EINVAL, "face tables: leaves need 0 <= xL < xR, yL < yR, zL < zR, f >= 0");
            const double V = ((b[1] - b[0]) * (b[3] - b[2])) * (b[5] - b[4]);
            sum += V * fl * std::fabs((b[0] + b[1]) / 2.0);
            cum[l] = sum;
        }
        if (!(sum > 0.0)) return fail(TITAN_EINVAL, "face tables: a face's distribution lets nothing in");
        flux[i] = sum;
        for (int64_t l = l0; l < l1; ++l) cum[l] = (l == l1 - 1) ? 1.0 : cum[l] / sum;
    }
    std::vector<double> frame(d->frame, d->frame + 9 * nt);
    std::vector<double> box(d->leaf_box, d->leaf_box + 6 * nleaf);
    cudaError_t e = upload_vec(&ctx->fd_buf[0], index);
    if (!e) e = upload_vec(&ctx->fd_buf[1], frame);
    if (!e) e = upload_vec(&ctx->fd_buf[2], side);
    if (!e) e = upload_vec(&ctx->fd_buf[3], flux);
    if (!e) e = upload_vec(&ctx->fd_buf[4], ptr);
    if (!e) e = upload_vec(&ctx->fd_buf[5], box);
    if (!e) e = upload_vec(&ctx->fd_buf[6], cum);
    if (e) {
        for (void*& p : ctx->fd_buf) {
            if (p) cudaFree(p);
            p = nullptr;
        }
        return fail(TITAN_ECUDA, std::string("face tables: ") + cudaGetErrorString(e));
    }
    return TITAN_OK;
}

namespace {
void drop_face_tally(titan_ctx* ctx) {
    for (void*& p : ctx->ft_buf) {
        if (p) cudaFree(p);
        p = nullptr;
    }
    ctx->ft_ntab = ctx->ft_nleaf = 0;
    ctx->ft_valid = false;
}
}  // namespace

int titan_set_mc_face_tally(titan_ctx* ctx, const titan_mc_face_tally* d) {
    if (!ctx) return fail(TITAN_EINVAL, "null argument");
    drop_face_tally(ctx);
    if (!d || d->nface == 0) return TITAN_OK;
    if (d->nface < 0 || !d->face || !d->side || !d->frame || !d->leaf_ptr || !d->leaf_box)
        return fail(TITAN_EINVAL, "face tallies: nface >= 0 and every array");
    const int64_t nf = ctx->nface, nt = d->nface;
    const Renumbering& R = ctx->R;
    if (d->leaf_ptr[0] != 0) return fail(TITAN_EINVAL, "face tallies: leaf_ptr[0] must be 0");
    const int64_t nleaf = d->leaf_ptr[nt];
    if (nleaf < nt || nleaf > INT32_MAX) return fail(TITAN_EINVAL, "face tallies: leaf_ptr[nface] out of range");
    std::vector<int32_t> index(nf, -1), face(nt), ptr(nt + 1, 0);
    std::vector<int8_t> side(nt);
    std::vector<double> bounds(6 * nt);
    std::vector<int32_t> c1(nf);
    CK(cudaMemcpy(c1.data(), ctx->d_face_c1, sizeof(int32_t) * nf, cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < nt; ++i) {
        const int32_t fo = d->face[i];
        if (fo < 0 || fo >= nf) return fail(TITAN_EINVAL, "face tallies: face id out of range");
        const int32_t f = R.face_o2n[fo];
        if (index[f] >= 0) return fail(TITAN_EINVAL, "face tallies: a face is listed twice");
        index[f] = (int32_t)i;
        face[i] = f;
        if (d->side[i] != 0 && d->side[i] != 1) return fail(TITAN_EINVAL, "face tallies: side is 0 or 1");
        if (d->side[i] == 1 && c1[f] < 0) return fail(TITAN_EINVAL, "face tallies: side 1 on a boundary face");
        side[i] = d->side[i];
        const int64_t l0 = d->leaf_ptr[i], l1 = d->leaf_ptr[i + 1];
        if (!(l1 > l0) || l1 > nleaf) return fail(TITAN_EINVAL, "face tallies: leaf_ptr must increase to leaf_ptr[nface]");
        ptr[i + 1] = (int32_t)l1;
        double* B = &bounds[6 * i];
        for (int k = 0; k < 6; k += 2) {
            B[k] = INFINITY;
            B[k + 1] = -INFINITY;
        }
        for (int64_t l = l0; l < l1; ++l) {
            const double* b = d->leaf_box + 6 * l;
            if (!(b[0] >= 0.0 && b[1] > b[0] && b[3] > b[2] && b[5] > b[4]) || !std::isfinite(b[1]) ||
                !std::isfinite(b[2]) || !std::isfinite(b[3]) || !std::isfinite(b[4]) || !std::isfinite(b[5]))
                return fail(TITAN_EINVAL, "face tallies: leaves need 0 <= xL < xR, yL < yR, zL < zR");
            for (int k = 0; k < 6; k += 2) {
                B[k] = std::min(B[k], b[k]);
                B[k + 1] = std::max(B[k + 1], b[k + 1]);
            }
        }
    }
    std::vector<double> frame(d->frame, d->frame + 9 * nt);
    std::vector<double> box(d->leaf_box, d->leaf_box + 6 * nleaf);
    cudaError_t e = upload_vec(&ctx->ft_buf[0], index);
    if (!e) e = upload_vec(&ctx->ft_buf[1], face);
    if (!e) e = upload_vec(&ctx->ft_buf[2], side);
    if (!e) e = upload_vec(&ctx->ft_buf[3], frame);
    if (!e) e = upload_vec(&ctx->ft_buf[4], bounds);
    if (!e) e = upload_vec(&ctx->ft_buf[5], ptr);
    if (!e) e = upload_vec(&ctx->ft_buf[6], box);
    if (!e) e = cudaMalloc(&ctx->ft_buf[7], sizeof(double) * nleaf);
    if (!e) e = cudaMalloc(&ctx->ft_buf[8], sizeof(double) * 3 * nt);
    if (!e) e = cudaMalloc(&ctx->ft_buf[9], sizeof(unsigned long long));
    if (e) {
        drop_face_tally(ctx);
        return fail(TITAN_ECUDA, std::string("face tallies: ") + cudaGetErrorString(e));
    }
    ctx->ft_ntab = nt;
    ctx->ft_nleaf = nleaf;
    return TITAN_OK;
}

int titan_get_mc_face_tally(titan_ctx* ctx, double* leaf_f, double* moments, int64_t* unplaced) {
    if (!ctx) return fail(TITAN_EINVAL, "null argument");
    if (!ctx->ft_valid) return fail(TITAN_EINVAL, "face tallies: no Monte-Carlo pass since they were set");
    if (leaf_f) CK(cudaMemcpy(leaf_f, ctx->ft_buf[7], sizeof(double) * ctx->ft_nleaf, cudaMemcpyDeviceToHost));
    if (moments) CK(cudaMemcpy(moments, ctx->ft_buf[8], sizeof(double) * 3 * ctx->ft_ntab, cudaMemcpyDeviceToHost));
    if (unplaced) {
        unsigned long long u = 0;
        CK(cudaMemcpy(&u, ctx->ft_buf[9], sizeof(u), cudaMemcpyDeviceToHost));
        *unplaced = (int64_t)u;
    }
    return TITAN_OK;
}

int titan_set_surface_motion(titan_ctx* ctx, const titan_surface_params* sp, int64_t nray, int32_t ray_len,
                             const int32_t* ray_nodes) {
    if (!ctx) return fail(TITAN_EINVAL, "null argument");
    drop_graph(ctx);
    drop_surface(ctx);
    if (!sp) return TITAN_OK;
    if (!ctx->prm.move) return fail(TITAN_EINVAL, "surface tracking needs a context created with move = 1");
    if (nray <= 0 || ray_len < 2 || !ray_nodes) return fail(TITAN_EINVAL, "rays: nray > 0, ray_len >= 2 and ids");
    const int64_t nf = ctx->nface, nn = ctx->nnode;
    const Renumbering& R = ctx->R;
    // mesh tables in device numbering
    std::vector<int8_t> surf(nf), ftype(nf);
    std::vector<int32_t> fnodes(4 * nf);
    CK(cudaMemcpy(surf.data(), ctx->d_face_surf, nf, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(ftype.data(), ctx->d_face_type, nf, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(fnodes.data(), ctx->d_face_nodes, sizeof(int32_t) * 4 * nf, cudaMemcpyDeviceToHost));
    auto moves = [&](int s) {
        return (s == 1 && sp->move_TS) || (s == 2 && sp->move_HP) || (s == 3 && sp->move_BS);
    };
    // surface neighbours of each surface face (Gran::grans_surf): faces of the
    // same surface across each edge
    std::map<std::tuple<int32_t, int32_t, int>, int> edges;
    auto edge = [&](int64_t f, int k) {
        int32_t a = fnodes[k * nf + f], b = fnodes[((k + 1) % 4) * nf + f];
        if (a > b) std::swap(a, b);
        return std::make_tuple(a, b, (int)surf[f]);
    };
    for (int64_t f = 0; f < nf; ++f)
        if (surf[f] >= 1 && surf[f] <= 3)
            for (int k = 0; k < 4; ++k) edges[edge(f, k)]++;
    std::vector<int8_t> node_surf(nn, 0);
    std::vector<std::vector<int32_t>> by_surf(4);
    for (int64_t f = 0; f < nf; ++f) {
        const int s = surf[f];
        if (s < 1 || s > 3) continue;
        for (int k = 0; k < 4; ++k) node_surf[fnodes[k * nf + f]] = (int8_t)s;
        if (!moves(s) || ftype[f] != 0) continue;
        if (s == 2) {
            int nb = 0;
            for (int k = 0; k < 4; ++k) nb += edges[edge(f, k)] - 1;
            if (nb < 4) continue;
        }
        by_surf[s].push_back((int32_t)f);
    }
    SurfaceDev S{};
    std::vector<int32_t> face_list;
    S.off[0] = S.off[1] = 0;
    for (int s = 1; s <= 3; ++s) {
        face_list.insert(face_list.end(), by_surf[s].begin(), by_surf[s].end());
        S.off[s + 1] = (int)face_list.size();
    }
    S.nlist = (int)face_list.size();
    // per moving surface node: its faces' list positions, ascending original face index
    std::vector<std::vector<std::pair<int32_t, int32_t>>> nf_of(nn);
    for (int pos = 0; pos < S.nlist; ++pos) {
        const int64_t f = face_list[pos];
        for (int k = 0; k < 4; ++k) nf_of[fnodes[k * nf + f]].push_back({R.face_n2o[f], pos});
    }
    std::vector<int32_t> node_id, node_ptr{0}, node_face;
    for (int64_t i = 0; i < nn; ++i) {
        if (!node_surf[i] || !moves(node_surf[i])) continue;
        auto& v = nf_of[i];
        std::sort(v.begin(), v.end());
        node_id.push_back((int32_t)i);
        for (auto& pr : v) node_face.push_back(pr.second);
        node_ptr.push_back((int32_t)node_face.size());
    }
    S.n_node = (int)node_id.size();
    // rays in device numbering, with the radii and directions of this layer
    std::vector<double> xyz(3 * nn);
    CK(cudaMemcpy(xyz.data(), ctx->layer[ctx->cur].xyz, sizeof(double) * 3 * nn, cudaMemcpyDeviceToHost));
    // smoothing: each moving node's surface neighbours (the nodes of its
    // surface's faces), ascending original id, and the fitted sphere centre
    std::vector<std::vector<int32_t>> faces_of(nn);
    for (int64_t f = 0; f < nf; ++f)
        if (surf[f] >= 1 && surf[f] <= 3)
            for (int k = 0; k < 4; ++k) faces_of[fnodes[k * nf + f]].push_back((int32_t)f);
    std::vector<signed char> sm_kind(S.n_node, 0);
    std::vector<double> sm_coef(S.n_node, 0.0), sm_centre(3 * (size_t)S.n_node, 0.0);
    std::vector<int32_t> nb_ptr{0}, nb_id;
    for (int i = 0; i < S.n_node; ++i) {
        const int32_t d = node_id[i];
        const int s = node_surf[d];
        const bool sphere = (s == 1 && sp->sglag_TS) || (s == 2 && sp->sglag_HP);
        const bool laplace = (s == 3 && sp->sglag_BS);
        std::vector<int32_t> nbs;
        if (sphere || laplace) {
            for (int32_t f : faces_of[d]) {
                if (surf[f] != s) continue;
                for (int k = 0; k < 4; ++k) {
                    const int32_t j = fnodes[k * nf + f];
                    if (j != d) nbs.push_back(j);
                }
            }
            std::sort(nbs.begin(), nbs.end(),
                      [&](int32_t x, int32_t y) { return R.node_n2o[x] < R.node_n2o[y]; });
            nbs.erase(std::unique(nbs.begin(), nbs.end()), nbs.end());
        }
        if (sphere && !nbs.empty()) {
            sm_kind[i] = 1;
            sm_coef[i] = (s == 1 ? sp->velocity_TS * sp->sglag_TS_k_sphere : sp->velocity_HP * sp->sglag_HP_k_sphere);
            std::vector<std::array<double, 3>> P;
            P.push_back({xyz[d], xyz[nn + d], xyz[2 * nn + d]});
            for (int32_t j : nbs) P.push_back({xyz[j], xyz[nn + j], xyz[2 * nn + j]});
            double c[3];
            fit_centre(P, c);
            for (int k = 0; k < 3; ++k) sm_centre[(size_t)k * S.n_node + i] = c[k];
        } else if (laplace) {
            sm_kind[i] = 2;
            sm_coef[i] = sp->velocity_BS * sp->sglag_BS_k;
        }
        if (sm_kind[i]) nb_id.insert(nb_id.end(), nbs.begin(), nbs.end());
        nb_ptr.push_back((int32_t)nb_id.size());
    }
    const int64_t L = ray_len;
    std::vector<int32_t> rn(nray * L);
    std::vector<double> r0(nray * L), dir(3 * nray);
    std::vector<uint8_t> anchor(nray * L), seen(nn, 0);
    std::vector<int2> seg(nray * L);
    for (int64_t r = 0; r < nray; ++r) {
        // a shorter ray ends at its first -1
        int64_t Lr = 0;
        while (Lr < L && ray_nodes[r * L + Lr] >= 0) ++Lr;
        if (Lr < 2) return fail(TITAN_EINVAL, "a ray needs at least two nodes");
        for (int64_t j = 0; j < L; ++j) {
            const int32_t o = ray_nodes[r * L + j];
            seg[r * L + j] = make_int2(-1, -1);
            if (j >= Lr) {
                if (o != -1) return fail(TITAN_EINVAL, "a ray's padding after its first -1 must be -1");
                rn[r * L + j] = -1;
                r0[r * L + j] = 0.0;
                continue;
            }
            if (o >= nn) return fail(TITAN_EINVAL, "ray node id out of range");
            const int32_t d = R.node_o2n[o];
            if (seen[d]++) return fail(TITAN_EINVAL, "a node lies on two rays, or twice on one");
            rn[r * L + j] = d;
            const double x = xyz[d], y = xyz[nn + d], z = xyz[2 * nn + d];
            r0[r * L + j] = std::sqrt(x * x + y * y + z * z);
            anchor[r * L + j] = (j == 0 || j == Lr - 1 || node_surf[d] != 0) ? 1 : 0;
        }
        for (int64_t a = 0, b = 1; b < Lr; ++b) {
            if (!anchor[r * L + b]) continue;
            for (int64_t j = a + 1; j < b; ++j) seg[r * L + j] = make_int2((int)a, (int)b);
            a = b;
        }
        const int32_t d0 = rn[r * L];
        const double x = xyz[d0], y = xyz[nn + d0], z = xyz[2 * nn + d0];
        const double n0 = std::sqrt(x * x + y * y + z * z);
        dir[3 * r] = x / n0;
        dir[3 * r + 1] = y / n0;
        dir[3 * r + 2] = z / n0;
    }
    S.nray = (int)nray;
    S.ray_len = ray_len;
    S.vel[1] = sp->velocity_TS;
    S.vel[2] = sp->velocity_HP;
    S.vel[3] = sp->velocity_BS;
    S.null_bn_on_hp = sp->null_bn_on_HP;
    cudaError_t e = upload_vec(&ctx->surf_buf[0], face_list);
    if (!e && S.nlist) e = cudaMalloc(&ctx->surf_buf[1], sizeof(double) * 3 * S.nlist);
    if (!e) e = upload_vec(&ctx->surf_buf[2], node_id);
    if (!e) e = upload_vec(&ctx->surf_buf[3], node_ptr);
    if (!e) e = upload_vec(&ctx->surf_buf[4], node_face);
    if (!e) e = upload_vec(&ctx->surf_buf[5], rn);
    if (!e) e = upload_vec(&ctx->surf_buf[6], r0);
    if (!e) e = upload_vec(&ctx->surf_buf[7], dir);
    if (!e) e = upload_vec(&ctx->surf_buf[8], seg);
    if (!e) e = upload_vec(&ctx->surf_buf[9], sm_kind);
    if (!e) e = upload_vec(&ctx->surf_buf[10], sm_coef);
    if (!e) e = upload_vec(&ctx->surf_buf[11], sm_centre);
    if (!e) e = upload_vec(&ctx->surf_buf[12], nb_ptr);
    if (!e) e = upload_vec(&ctx->surf_buf[13], nb_id);
    if (!e && sp->hp_tail) {
        std::vector<signed char> tail(S.n_node);
        for (int i = 0; i < S.n_node; ++i) tail[i] = node_surf[node_id[i]] == 2 ? 1 : 0;
        e = upload_vec(&ctx->surf_buf[14], tail);
    }
    if (e) {
        drop_surface(ctx);
        return fail(TITAN_ECUDA, std::string("surface tables: ") + cudaGetErrorString(e));
    }
    S.face_list = (const int*)ctx->surf_buf[0];
    S.vf = (double*)ctx->surf_buf[1];
    S.node_id = (const int*)ctx->surf_buf[2];
    S.node_ptr = (const int*)ctx->surf_buf[3];
    S.node_face = (const int*)ctx->surf_buf[4];
    S.ray_nodes = (const int*)ctx->surf_buf[5];
    S.ray_r0 = (const double*)ctx->surf_buf[6];
    S.ray_dir = (const double*)ctx->surf_buf[7];
    S.ray_seg = (const int2*)ctx->surf_buf[8];
    S.sm_kind = (const signed char*)ctx->surf_buf[9];
    S.sm_coef = (const double*)ctx->surf_buf[10];
    S.sm_centre = (const double*)ctx->surf_buf[11];
    S.nb_ptr = (const int*)ctx->surf_buf[12];
    S.nb_id = (const int*)ctx->surf_buf[13];
    S.node_tail = (const signed char*)ctx->surf_buf[14];
    ctx->surf = S;
    ctx->use_surface = true;
    ctx->h_ray_nodes = std::move(rn);
    ctx->h_node_surf = std::move(node_surf);
    return TITAN_OK;
}

int titan_set_ray_law(titan_ctx* ctx, const titan_ray_law* law) {
    if (!ctx) return fail(TITAN_EINVAL, "null argument");
    if (!ctx->use_surface) return fail(TITAN_EINVAL, "the ray law needs titan_set_surface_motion first");
    drop_graph(ctx);
    if (!law) {
        ctx->surf.law = RayLaw{};
        return TITAN_OK;
    }
    RayLaw g{};
    g.on = 1;
    g.M0 = law->M0;
    g.M1 = law->M1;
    g.M11 = law->M11;
    g.M2 = law->M2;
    g.M3 = law->M3;
    g.M4 = law->M4;
    g.R0 = law->R0;
    g.R1 = law->R1;
    g.R5 = law->R5;
    g.da1 = law->da1;
    g.da2 = law->da2;
    g.da3 = law->da3;
    g.da4 = law->da4;
    g.da5 = law->da5;
    if (g.M0 < 1 || g.M1 < 0 || g.M11 < 0 || g.M2 < g.M11 || g.M3 < 0 || g.M4 < 0)
        return fail(TITAN_EINVAL, "ray law: M0 >= 1, M1, M3, M4 >= 0 and 0 <= M11 <= M2");
    const double v[] = {g.R0, g.R1, g.R5, g.da1, g.da2, g.da3, g.da4, g.da5};
    for (double x : v)
        if (!std::isfinite(x)) return fail(TITAN_EINVAL, "ray law: radii and da1..da5 must be finite");
    const int L = ctx->surf.ray_len;
    if (g.length() != L)
        return fail(TITAN_EINVAL, "ray law: every ray needs M0 + M1 + M2 + M3 + M4 + 5 nodes");
    const int slot[3] = {g.ts_slot(), g.hp_slot(), g.bs_slot()};
    for (int64_t r = 0; r < ctx->surf.nray; ++r)
        for (int k = 0; k < 3; ++k) {
            const int32_t d = ctx->h_ray_nodes[r * L + slot[k]];
            if (d < 0 || ctx->h_ray_nodes[r * L + L - 1] < 0)
                return fail(TITAN_EINVAL, "ray law: a ray is shorter than the law's length");
            if (ctx->h_node_surf[d] != k + 1) {
                char buf[160];
                snprintf(buf, sizeof buf, "ray law: node %d of ray %lld is not on the %s surface", slot[k],
                         (long long)r, k == 0 ? "TS" : k == 1 ? "HP" : "BS");
                return fail(TITAN_EINVAL, buf);
            }
        }
    ctx->surf.law = g;
    return TITAN_OK;
}

int titan_set_closure_overlap(titan_ctx* ctx, int32_t on) {
    if (!ctx) return fail(TITAN_EINVAL, "null argument");
    ctx->overlap_closure = on != 0;
    drop_graph(ctx);
    return TITAN_OK;
}

int titan_set_tuning(titan_ctx* ctx, int32_t face_variant, int32_t cell_variant) {
    if (!ctx) return fail(TITAN_EINVAL, "null argument");
    if (face_variant < 0 || face_variant >= kFaceVariants || cell_variant < 0 || cell_variant >= kCellVariants)
        return fail(TITAN_EINVAL, "variant out of range");
    if (kCellVariant[cell_variant].overflow > 0 && !ctx->d_owner_start)
        return fail(TITAN_EINVAL, "staged cell update needs the faces sorted by cells[0]");
    ctx->face_variant = face_variant;
    ctx->cell_variant = cell_variant;
    drop_graph(ctx);
    return TITAN_OK;
}

int titan_get_tuning(titan_ctx* ctx, int32_t* face_variant, int32_t* cell_variant, int32_t* face_block,
                     int32_t* face_min_blocks, int32_t* cell_block) {
    if (!ctx) return fail(TITAN_EINVAL, "null argument");
    if (face_variant) *face_variant = ctx->face_variant;
    if (cell_variant) *cell_variant = ctx->cell_variant;
    if (face_block) *face_block = kFaceVariant[ctx->face_variant].block;
    if (face_min_blocks) *face_min_blocks = kFaceVariant[ctx->face_variant].min_blocks;
    if (cell_block) *cell_block = kCellVariant[ctx->cell_variant].block;
    return TITAN_OK;
}

int titan_autotune(titan_ctx* ctx, int32_t reps, const char* cache_path) {
    if (!ctx || reps <= 0) return fail(TITAN_EINVAL, "bad argument");
    const int src = step_source_mode(ctx);
    char key[256];
    snprintf(key, sizeof key, "sm_100a cells=%lld faces=%lld move=%d flux=%d npassive=%d src=%d tvd=%d",
             (long long)ctx->ncell, (long long)ctx->nface, ctx->prm.move, ctx->prm.flux_precision,
             ctx->prm.npassive, src, ctx->P.tvd);
    if (cache_path) {
        FILE* f = fopen(cache_path, "r");
        if (f) {
            char line[512];
            while (fgets(line, sizeof line, f)) {
                char* bar = strchr(line, '|');
                if (!bar) continue;
                *bar = 0;
                int fv = -1, cv = -1;
                if (strcmp(line, key) == 0 && sscanf(bar + 1, "%d %d", &fv, &cv) == 2 && fv >= 0 &&
                    fv < kFaceVariants && cv >= 0 && cv < kCellVariants) {
                    fclose(f);
                    return titan_set_tuning(ctx, fv, cv);
                }
            }
            fclose(f);
        }
    }
    cudaStream_t s = ctx->stream;
    const MeshView M = ctx->view();
    const bool move = ctx->prm.move != 0;
    const int nxt = ctx->cur ^ 1;
    // the next layer = the current one, so every input the kernels read is valid
    if (move)
        CK(cudaMemcpyAsync(ctx->layer[nxt].xyz, ctx->layer[ctx->cur].xyz, sizeof(double) * 3 * ctx->nnode,
                           cudaMemcpyDeviceToDevice, s));
    DevStatus init{};
    init.dt = 1e-5;
    init.dt_next_bits = 0x4197D78400000000ull;
    FaceArgs fa;
    fa.M = M;
    fa.P = ctx->P;
    fa.L1 = ctx->layer[ctx->cur];
    fa.xyz2 = ctx->layer[nxt].xyz;
    fa.state = ctx->d_state[ctx->scur];
    fa.flux = ctx->d_flux;
    fa.st = ctx->d_status;
    CellArgs ca;
    ca.M = M;
    ca.P = ctx->P;
    ca.vol1 = ctx->layer[ctx->cur].vol;
    ca.vol2 = ctx->layer[ctx->cur].vol;
    ca.L2 = ctx->layer[nxt];
    ca.state = ctx->d_state[ctx->scur];
    ca.state2 = ctx->d_state[ctx->scur ^ 1];
    ca.flux = ctx->d_flux;
    ca.hfl = ctx->d_hfl;
    ca.src = ctx->d_src;
    ca.cl = closure_cell(ctx);
    ca.st = ctx->d_status;
    ca.owner_start = ctx->d_owner_start;
    const int nk = ctx->prm.npassive;
    // the timed cell updates write the closure's next inputs from a state the
    // context does not keep: they are formed again before the next step
    ctx->cl_valid = false;
    auto time_it = [&](auto launch, float* ms_out) -> cudaError_t {
        std::memcpy(ctx->h_status, &init, sizeof(DevStatus));
        cudaError_t e = cudaMemcpyAsync(ctx->d_status, ctx->h_status, sizeof(DevStatus), cudaMemcpyHostToDevice, s);
        if (!e) e = launch();
        if (!e) e = cudaEventRecord(ctx->ev[0], s);
        for (int r = 0; r < reps && !e; ++r) e = launch();
        if (!e) e = cudaEventRecord(ctx->ev[1], s);
        if (!e) e = cudaEventSynchronize(ctx->ev[1]);
        if (!e) e = cudaEventElapsedTime(ms_out, ctx->ev[0], ctx->ev[1]);
        return e;
    };
    float best = 1e30f;
    int best_fv = 0, best_cv = 0;
    float fms[kFaceVariants], cms[kCellVariants];
    for (int v = 0; v < kFaceVariants; ++v) {
        CK(time_it([&] { return face_launch(ctx, fa, nk, move, v, s); }, &fms[v]));
        if (fms[v] < best) {
            best = fms[v];
            best_fv = v;
        }
    }
    best = 1e30f;
    for (int v = 0; v < kCellVariants; ++v) {
        cms[v] = 1e30f;
        if (kCellVariant[v].overflow > 0 && !ctx->d_owner_start) continue;
        CK(time_it([&] { return launch_cell_update(ca, nk, move, src, v, s); }, &cms[v]));
        if (cms[v] < best) {
            best = cms[v];
            best_cv = v;
        }
    }
    CK(cudaStreamSynchronize(s));
    const int rc = titan_set_tuning(ctx, best_fv, best_cv);
    if (rc) return rc;
    if (cache_path) {
        FILE* f = fopen(cache_path, "a");
        if (f) {
            fprintf(f, "%s|%d %d  # face ms/launch:", key, best_fv, best_cv);
            for (int v = 0; v < kFaceVariants; ++v) fprintf(f, " %.4f", fms[v] / reps);
            fprintf(f, "  cell:");
            for (int v = 0; v < kCellVariants; ++v) fprintf(f, " %.4f", cms[v] / reps);
            fprintf(f, "\n");
            fclose(f);
        }
    }
    return TITAN_OK;
}

void* titan_stream(titan_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int titan_set_profiling(titan_ctx* ctx, int32_t on) {
    if (!ctx) return fail(TITAN_EINVAL, "null argument");
    ctx->profiling = on != 0;
    if (on) ctx->clocks.clear();
    return TITAN_OK;
}

int titan_kernel_times(titan_ctx* ctx, const char** names, double* total_ms, int64_t* launches, int32_t cap) {
    if (!ctx) return fail(TITAN_EINVAL, "null argument");
    // names point into the map's keys: valid until profiling is switched on again
    int i = 0;
    for (auto& kv : ctx->clocks) {
        if (i >= cap) break;
        if (names) names[i] = kv.first.c_str();
        if (total_ms) total_ms[i] = kv.second.ms;
        if (launches) launches[i] = kv.second.launches;
        ++i;
    }
    return i;
}

int64_t titan_device_bytes(titan_ctx* ctx) { return ctx ? ctx->dev_bytes : 0; }

}  // extern "C"
