// Surface-tracking node motion (-fmad=false, like the FP64 step): the
// reference's Setka::Culc_Velocity_surface (TITAN/source/Setka_move.cpp:111-1358)
// and Luch::dvigenie (Luch.cpp:6-739) for meshes whose rays are straight lines
// of nodes.
//
//  1. Per moving surface, in the reference's order TS, HP, BS (so BS sees the
//     HP cells' B as null_bn_on_HP left it): one thread per surface face forms
//     the face's geometry on this layer and its reconstructed states, solves
//     the Riemann problem at w = 0 and keeps velocity_X * ds * n, ds = dsl on
//     TS, dsc on HP (the exact gas-dynamic solver with bn_in_p_on_HP), dsr on
//     BS (Setka_move.cpp:128-447). HP faces with fewer than four surface
//     neighbours are left out of the list (:192).
//  2. One thread per surface node: the mean of its faces' contributions,
//     summed in ascending original face order, and the move
//     x' = x + (V . x/|x|) dt x/|x| (:1213-1265); with hp_tail an HP node
//     with x < 0 moves along (0, y, z) instead (:1237-1247).
//  3. One thread per ray node: every node between two anchors (the ray's ends
//     and its surface nodes) keeps its initial fraction of that segment, on
//     the ray's direction; or, with the A_Luch law (Luch.cpp:9-152), takes the
//     radius that law gives it from the ray's TS, HP and BS radii.
// With smoothing on, a node's mean also takes one smoothing term (sglag_*): toward
// the sphere fitted through it and its neighbours (TS, HP) or toward the mean of
// them (BS).
#include "launch.h"
#include "step_kernels.cuh"
#include "surface.h"

namespace titan {
namespace surf {

// Surfaces s_lo..s_hi in one launch (their list positions are contiguous).
template <int NK, bool TVD>
__global__ void __launch_bounds__(128) speed_kernel(FaceArgs a, SurfaceDev S, double* state_rw, int s_lo, int s_hi) {
    const int pos = S.off[s_lo] + blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= S.off[s_hi + 1] || a.st->err_kind != 0) return;
    int s = s_lo;
    while (pos >= S.off[s + 1]) ++s;
    const MeshView& M = a.M;
    const Params& P = a.P;
    const int nf = M.nface, nc = M.ncell, nn = M.nnode;
    const int f = S.face_list[pos];
    const int c0 = M.face_c0[f], c1 = M.face_c1[f];
    // this layer's geometry of the face (Gran::Culc_measure)
    double X[4][3];
#pragma unroll
    for (int k = 0; k < 4; ++k) load_node(a.L1.xyz, nn, M.face_nodes[k * nf + f], X[k]);
    double cA[3], cB[3];
    load_cc(a.L1.cc, nc, c0, cA);
    load_cc(a.L1.cc, nc, c1, cB);
    const FaceGeom g = face_geometry(X, cA, cB);
    const double n[3] = {g.n[0], g.n[1], g.n[2]};
    double gc[3] = {g.c[0], g.c[1], g.c[2]};
    const bool nullbn = (s == 2 && S.null_bn_on_hp);
    if (nullbn) {
        // the cells' own B loses its normal part (Setka_move.cpp:196-224)
        const int cs[2] = {c0, c1};
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            double* bx = state_rw + 5 * nc + cs[j];
            double* by = state_rw + 6 * nc + cs[j];
            double* bz = state_rw + 7 * nc + cs[j];
            const double dtpr = n[0] * *bx + n[1] * *by + n[2] * *bz;
            *bx -= dtpr * n[0];
            *by -= dtpr * n[1];
            *bz -= dtpr * n[2];
        }
    }
    double Ls[NV], Rs[NV];
    face_states<NK, true, TVD, false>(a, f, 0, c0, n, gc, Ls, Rs);
    int method;
    if (P.method_policy == 1) {
        const double bb =
            ((Ls[5] * Ls[5] + Ls[6] * Ls[6] + Ls[7] * Ls[7]) + (Rs[5] * Rs[5] + Rs[6] * Rs[6] + Rs[7] * Rs[7])) / 2.0;
        const double pp = (Ls[4] + Rs[4]) / 2.0;
        method = (bb / (4.0 * kPi) / (2.0 * pp) > P.beta_switch) ? 3 : 2;
    } else {
        method = M.face_method[f];
    }
    if (nullbn) {
        // and so do the face states (:279-295)
        double* qs[2] = {Ls, Rs};
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            double* q = qs[j];
            const double dtpr = n[0] * q[5] + n[1] * q[6] + n[2] * q[7];
            q[5] -= dtpr * n[0];
            q[6] -= dtpr * n[1];
            q[7] -= dtpr * n[2];
        }
    }
    double dsl = 0.0, dsc = 0.0, dsr = 0.0;
    if (s == 2 && P.bn_in_p_on_hp) {
        const GodunovFlux gd = godunov_hp_face(n[0], n[1], n[2], 0.0, Ls[0], Ls[1], Ls[2], Ls[3], Ls[4], Ls[5], Ls[6],
                                               Ls[7], Rs[0], Rs[1], Rs[2], Rs[3], Rs[4], Rs[5], Rs[6], Rs[7], 0, P.gamma);
        if (gd.rc) record_error(a.st, 14 + gd.rc, f);
        dsl = gd.dsl;
        dsc = gd.dsc;
        dsr = gd.dsr;
    } else {
        double qd[8];
        RiemannFlags fl;
        fl.null_bn = false;
        fl.left_ydar = false;
        fl.contact = false;
        fl.n_disc = 0;
        const int rc = riemann_flux<double, 0>(method, n, 0.0, Ls, Rs, nullptr, nullptr, qd, nullptr, dsl, dsc, dsr,
                                               fl, P.gamma);
        if (rc) record_error(a.st, 10 + rc, f);
    }
    if (s == 2 && (isnan(dsc) || (dsc != 0.0 && fabs(dsc) < 2.2250738585072014e-308))) record_error(a.st, 19, f);
    const double d = (s == 1) ? dsl : ((s == 2) ? dsc : dsr);
    const double vd = S.vel[s] * d;
#pragma unroll
    for (int k = 0; k < 3; ++k) S.vf[k * S.nlist + pos] = vd * n[k];
}

__global__ void node_kernel(FaceArgs a, SurfaceDev S) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.n_node || a.st->err_kind != 0) return;
    const int nn = a.M.nnode;
    const int id = S.node_id[i];
    double v[3] = {0.0, 0.0, 0.0};
    const int j0 = S.node_ptr[i], j1 = S.node_ptr[i + 1];
    for (int j = j0; j < j1; ++j) {
        const int pos = S.node_face[j];
#pragma unroll
        for (int k = 0; k < 3; ++k) v[k] += S.vf[k * S.nlist + pos];
    }
    int num = j1 - j0;
    double A[3];
    load_node(a.L1.xyz, nn, id, A);
    const double time = a.st->dt;
    const int kind = S.sm_kind[i];
    if (kind) {
        // smoothing (Setka_move.cpp:454-1211): one more term of the mean
        const int b0 = S.nb_ptr[i], b1 = S.nb_ptr[i + 1], nb = b1 - b0;
        const double coef = S.sm_coef[i];
        if (kind == 1) {
            // toward the sphere fitted at set-up through the node and its neighbours
            const double B[3] = {S.sm_centre[i], S.sm_centre[S.n_node + i], S.sm_centre[2 * S.n_node + i]};
            const double rr = sqrt((A[0] - B[0]) * (A[0] - B[0]) + (A[1] - B[1]) * (A[1] - B[1]) +
                                   (A[2] - B[2]) * (A[2] - B[2]));
            double r = 0.0;
            for (int j = b0; j < b1; ++j) {
                double X[3];
                load_node(a.L1.xyz, nn, S.nb_id[j], X);
                r += sqrt((X[0] - B[0]) * (X[0] - B[0]) + (X[1] - B[1]) * (X[1] - B[1]) +
                          (X[2] - B[2]) * (X[2] - B[2]));
            }
            r /= nb;
            const double kk = r / rr;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const double b2 = kk * (A[k] - B[k]) + B[k];
                v[k] += coef * (b2 - A[k]) / time;
            }
            ++num;
        } else if (nb > 5) {
            // toward the mean of the node and its neighbours
            double B[3] = {A[0], A[1], A[2]};
            for (int j = b0; j < b1; ++j) {
                double X[3];
                load_node(a.L1.xyz, nn, S.nb_id[j], X);
#pragma unroll
                for (int k = 0; k < 3; ++k) B[k] += X[k];
            }
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                B[k] /= (nb + 1.0);
                v[k] += coef * (B[k] - A[k]) / time;
            }
            ++num;
        }
    }
    if (num > 0) {
#pragma unroll
        for (int k = 0; k < 3; ++k) v[k] /= num;
    }
    // the direction of motion: x / |x|, or (0, y, z) normalised for an HP node
    // of the heliotail (x < 0) with hp_tail (Setka_move.cpp:1237-1247); a node
    // on the x axis keeps the zero vector, as Eigen's normalize() leaves it,
    // and stays
    double B[3];
    if (S.node_tail && S.node_tail[i] && A[0] < 0.0) {
        const double bn = sqrt(A[1] * A[1] + A[2] * A[2]);
        B[0] = 0.0;
        B[1] = bn > 0.0 ? A[1] / bn : 0.0;
        B[2] = bn > 0.0 ? A[2] / bn : 0.0;
    } else {
        const double an = sqrt(A[0] * A[0] + A[1] * A[1] + A[2] * A[2]);
        B[0] = A[0] / an;
        B[1] = A[1] / an;
        B[2] = A[2] / an;
    }
    const double vb = v[0] * B[0] + v[1] * B[1] + v[2] * B[2];
    double* x2 = const_cast<double*>(a.xyz2);
#pragma unroll
    for (int k = 0; k < 3; ++k) x2[k * nn + id] = A[k] + vb * time * B[k];
}

__device__ __forceinline__ double sq(double x) { return x * x; }

// Radius of slot j of a ray under the A_Luch law, from the current radii R2,
// R3, R4 of its TS, HP and BS nodes, with the reference's expressions
// (Luch.cpp:17-152); false for the slots the law leaves where they are (the
// R1 node and the three surface nodes).
__device__ bool a_luch_radius(const RayLaw& g, int j, double R2, double R3, double R4, double* r) {
    const int M0 = g.M0, M1 = g.M1, M11 = g.M11, M2 = g.M2, M3 = g.M3, M4 = g.M4;
    const double R0 = g.R0, R1 = g.R1, R5 = g.R5;
    if (j < M0) {
        *r = R0 + j * (R1 - R0) / M0;
        return true;
    }
    int num = M0 + 1;
    if (j < num) return false;
    if (j < num + M1) {
        *r = R1 + (j - num + 1) * (R2 - R1) / (M1 + 1);
        return true;
    }
    num += M1 + 1;
    if (j < num) return false;
    const double dr = (R2 - R1) / (M1 + 1);
    if (j < num + M11) {
        *r = R2 + dr * (j - num + 1);
        return true;
    }
    num += M11;
    if (j < num + (M2 - M11)) {
        const double a = g.da1, b = g.da2;
        const double s = (j - num + 1.0) / (M2 - M11 + 1.0);
        const double ss = s * (a * sq(1.0 - 3.0 * s + 2.0 * sq(s)) +
                               s * (7.0 + b * sq(1.0 - 2.0 * s) * (-1.0 + s) -
                                    2.0 * s * (9.0 + 2.0 * s * (-5.0 + 2.0 * s))));
        *r = R2 + dr * M11 + (R3 - R2 - dr * M11) * ss;
        return true;
    }
    num += (M2 - M11) + 1;
    if (j < num) return false;
    if (j < num + M3) {
        const double a = g.da3, b = g.da4;
        const double s = (j - num + 1.0) / (M3 + 1.0);
        const double ss = s * (a - (2.0 * a + b - 3.0) * s + (a + b - 2.0) * s * s);
        *r = R3 + (R4 - R3) * ss;
        return true;
    }
    num += M3 + 1;
    if (j < num) return false;
    if (j < num + M4) {
        const double a = g.da5, b = 2.0;
        const double s = (j - num + 1.0) / (M4 + 1.0);
        const double ss = a * s - (3.0 * a + b - 4.0) * s * s * s + (2.0 * a + b - 3.0) * s * s * s * s;
        *r = R4 + (R5 - R4) * ss;
        return true;
    }
    *r = R5;
    return true;
}

__device__ __forceinline__ double node_radius(const double* xyz, int nn, int id) {
    double x[3];
    load_node(xyz, nn, id, x);
    return sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
}

// One thread per ray slot: a node that is not an anchor takes its place
// between the anchors around it (ray_seg: their slots, set up once), or, with
// the A_Luch law, the place the law gives it from the ray's surface nodes.
__global__ void ray_kernel(FaceArgs a, SurfaceDev S) {
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q >= (long long)S.nray * S.ray_len || a.st->err_kind != 0) return;
    if (S.law.on) {
        const int L = S.ray_len, nn = a.M.nnode;
        const int r = (int)(q / L), j = (int)(q % L);
        const int* rn = S.ray_nodes + (long long)r * L;
        const double R2 = node_radius(a.xyz2, nn, rn[S.law.ts_slot()]);
        const double R3 = node_radius(a.xyz2, nn, rn[S.law.hp_slot()]);
        const double R4 = node_radius(a.xyz2, nn, rn[S.law.bs_slot()]);
        double rj;
        if (!a_luch_radius(S.law, j, R2, R3, R4, &rj)) return;
        double* x2 = const_cast<double*>(a.xyz2);
#pragma unroll
        for (int k = 0; k < 3; ++k) x2[k * nn + rn[j]] = rj * S.ray_dir[3 * r + k];
        return;
    }
    const int2 seg = S.ray_seg[q];
    if (seg.x < 0) return;  // an anchor
    const int nn = a.M.nnode, L = S.ray_len;
    const int r = (int)(q / L);
    const long long base = (long long)r * L;
    const double* x2c = a.xyz2;
    double xa[3], xb[3];
    load_node(x2c, nn, S.ray_nodes[base + seg.x], xa);
    load_node(x2c, nn, S.ray_nodes[base + seg.y], xb);
    const double ra = sqrt(xa[0] * xa[0] + xa[1] * xa[1] + xa[2] * xa[2]);
    const double rb = sqrt(xb[0] * xb[0] + xb[1] * xb[1] + xb[2] * xb[2]);
    const double r0a = S.ray_r0[base + seg.x], r0b = S.ray_r0[base + seg.y];
    const double rj = ra + (S.ray_r0[q] - r0a) / (r0b - r0a) * (rb - ra);
    double* x2 = const_cast<double*>(a.xyz2);
    const int id = S.ray_nodes[q];
#pragma unroll
    for (int k = 0; k < 3; ++k) x2[k * nn + id] = rj * S.ray_dir[3 * r + k];
}

}  // namespace surf

template <int NK, bool TVD>
static void launch_speeds(const FaceArgs& fa, double* state_rw, const SurfaceDev& S, cudaStream_t s) {
    auto run = [&](int lo, int hi) {
        const int n = S.off[hi + 1] - S.off[lo];
        if (n > 0) surf::speed_kernel<NK, TVD><<<blocks_for(n, 128), 128, 0, s>>>(fa, S, state_rw, lo, hi);
    };
    if (S.null_bn_on_hp) {
        // HP edits the cells' B: TS before it, BS after it, as the reference runs them
        for (int sf = 1; sf <= 3; ++sf) run(sf, sf);
    } else {
        run(1, 3);
    }
}

cudaError_t launch_surface_motion(const FaceArgs& fa, double* state_rw, const SurfaceDev& S, int nk, bool tvd,
                                  cudaStream_t s) {
    const int nn = fa.M.nnode;
    // nodes that neither a surface nor a ray moves keep their place
    cudaError_t e = cudaMemcpyAsync(const_cast<double*>(fa.xyz2), fa.L1.xyz, sizeof(double) * 3 * (size_t)nn,
                                    cudaMemcpyDeviceToDevice, s);
    if (e) return e;
    if (nk == 0 && !tvd) launch_speeds<0, false>(fa, state_rw, S, s);
    else if (nk == 0 && tvd) launch_speeds<0, true>(fa, state_rw, S, s);
    else if (nk == 2 && !tvd) launch_speeds<2, false>(fa, state_rw, S, s);
    else if (nk == 2 && tvd) launch_speeds<2, true>(fa, state_rw, S, s);
    else return cudaErrorInvalidValue;
    if (S.n_node > 0) surf::node_kernel<<<blocks_for(S.n_node, 128), 128, 0, s>>>(fa, S);
    if (S.nray > 0) surf::ray_kernel<<<blocks_for((long long)S.nray * S.ray_len, 256), 256, 0, s>>>(fa, S);
    return cudaGetLastError();
}

}  // namespace titan
