// Kernels of one explicit plasma time step on the SFC-renumbered mesh.
//
//   move_nodes      prescribed radial node motion (ALE), x' = x + dt*v(t)
//   cell_geometry   cell centre (mean of 8 nodes) and volume (12 tetrahedra)
//   face_geometry   face centre, area (2 triangles), oriented normal, half
//                   centre distance
//   face_flux<R>    reconstruction + Riemann flux in precision R, flux*area,
//                   Powell PdivB, CFL candidate -> warp/block min -> atomicMin
//   cell_update     deterministic gather of the 6 face fluxes in the cell's
//                   own face order (no atomics), conservative update with the
//                   ALE volume ratio, sources, Zone_2 dissipation, floors; the
//                   last block rolls the CFL dt over to the next step
//
// The arithmetic restates TITAN's Setka::Go plasma loops
// (TITAN/source/Setka_physics.cpp:1589-2028), Setka::Culc_Gran_Potok (:2280-2571),
// Setka::Snos_on_Gran (Setka_gran_snos.cpp:3-180, :737-1071), the geometry of
// Gran::Culc_measure / Cell::Culc_center / Cell::Culc_volume (Gran.cpp:112-218,
// Cell.cpp:909-1007) and Gran::culc_velosity (Gran.cpp:571-589), in the same
// expression order, so the FP64 instantiation (compiled with -fmad=false)
// reproduces the reference's rounding.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "godunov.cuh"
#include "riemann.cuh"
#include "step_types.h"

namespace titan {

__device__ __forceinline__ void record_error(DevStatus* st, int kind, int index) {
    if (atomicCAS(&st->err_kind, 0, kind) == 0) st->err_index = index;
}

// ---------------------------------------------------------------------------
// Node motion (ALE): the synthetic radial motion of the heliosphere shell.
// ---------------------------------------------------------------------------
static __global__ void move_nodes_kernel(MeshView M, Params P, const double* __restrict__ xyz1, double* __restrict__ xyz2,
                                  const DevStatus* __restrict__ st) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= M.nnode) return;
    const int nn = M.nnode;
    const double x = xyz1[i], y = xyz1[nn + i], z = xyz1[2 * nn + i];
    const double amp = M.node_amp ? M.node_amp[i] : 0.0;
    if (amp == 0.0) {
        xyz2[i] = x;
        xyz2[nn + i] = y;
        xyz2[2 * nn + i] = z;
        return;
    }
    const double time = st->dt, t = st->t;
    const double r = sqrt(x * x + y * y + z * z);
    const double v = amp * sin(P.omega * t + M.node_phase[i]);
    const double s = time * v / r;
    xyz2[i] = x + s * x;
    xyz2[nn + i] = y + s * y;
    xyz2[2 * nn + i] = z + s * z;
}

__device__ __forceinline__ double tri_area(double ax, double ay, double az, double bx, double by, double bz,
                                           double cx, double cy, double cz) {
    const double v1x = bx - ax, v1y = by - ay, v1z = bz - az;
    const double v2x = cx - ax, v2y = cy - ay, v2z = cz - az;
    const double x = v1y * v2z - v1z * v2y;
    const double y = v1z * v2x - v1x * v2z;
    const double z = v1x * v2y - v1y * v2x;
    return 0.5 * sqrt(x * x + y * y + z * z);
}

__device__ __forceinline__ double tet_vol(const double* a, const double* b, const double* c, const double* d) {
    const double abx = b[0] - a[0], aby = b[1] - a[1], abz = b[2] - a[2];
    const double acx = c[0] - a[0], acy = c[1] - a[1], acz = c[2] - a[2];
    const double adx = d[0] - a[0], ady = d[1] - a[1], adz = d[2] - a[2];
    const double x = aby * acz - abz * acy;
    const double y = abz * acx - abx * acz;
    const double z = abx * acy - aby * acx;
    return fabs(x * adx + y * ady + z * adz) / 6.0;
}

__device__ __forceinline__ void load_node(const double* xyz, int nn, int i, double* p) {
    p[0] = xyz[i];
    p[1] = xyz[nn + i];
    p[2] = xyz[2 * nn + i];
}

// Cell centre (Cell.cpp:909-930) and volume by method 1 (Cell.cpp:958-1001):
// two tetrahedra (C, P0, P1, P2) and (C, P0, P3, P2) per face, in face order.
// P(s, k) returns node k of face slot s.
template <typename NodeOf>
__device__ __forceinline__ double cell_volume(const double C[3], NodeOf P) {
    double V = 0.0;
#pragma unroll
    for (int s = 0; s < 6; ++s) {
        double P0[3], P1[3], P2[3], P3[3];
        P(s, 0, P0);
        P(s, 1, P1);
        P(s, 2, P2);
        P(s, 3, P3);
        V += tet_vol(C, P0, P1, P2);
        V += tet_vol(C, P0, P3, P2);
    }
    return V;
}

__device__ __forceinline__ void cell_centre(const double X[8][3], double C[3]) {
    double x = 0.0, y = 0.0, z = 0.0;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        x += X[k][0];
        y += X[k][1];
        z += X[k][2];
    }
    C[0] = x / 8;
    C[1] = y / 8;
    C[2] = z / 8;
}

static __global__ void cell_geometry_kernel(MeshView M, Layer L) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= M.ncell) return;
    const int nc = M.ncell, nn = M.nnode, nf = M.nface;
    double X[8][3];
#pragma unroll
    for (int k = 0; k < 8; ++k) load_node(L.xyz, nn, M.cell_nodes[k * nc + c], X[k]);
    double C[3];
    cell_centre(X, C);
    L.cc[c] = C[0];
    L.cc[nc + c] = C[1];
    L.cc[2 * nc + c] = C[2];
    L.vol[c] = cell_volume(C, [&](int s, int k, double* p) {
        const int f = M.cell_faces[s * nc + c] & 0x7fffffff;
        load_node(L.xyz, nn, M.face_nodes[k * nf + f], p);
    });
}

struct FaceGeom {
    double c[3];  // centre
    double n[3];  // unit normal from cells[0] to cells[1]
    double area;
    double half_dist;
};

// Face centre, area (2 triangles), normal from edge midpoints oriented from
// cells[0] to cells[1] (Gran.cpp:112-218) and half the distance between the
// two cell centres used by the CFL estimate (Setka_physics.cpp:2298-2307).
__device__ __forceinline__ FaceGeom face_geometry(const double P[4][3], const double c0[3], const double* c1) {
    FaceGeom g;
    double xc = 0.0, yc = 0.0, zc = 0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        xc += P[k][0];
        yc += P[k][1];
        zc += P[k][2];
    }
    xc /= 4;
    yc /= 4;
    zc /= 4;
    g.c[0] = xc;
    g.c[1] = yc;
    g.c[2] = zc;
    double S = 0.0;
    S += tri_area(P[0][0], P[0][1], P[0][2], P[1][0], P[1][1], P[1][2], P[2][0], P[2][1], P[2][2]);
    S += tri_area(P[0][0], P[0][1], P[0][2], P[3][0], P[3][1], P[3][2], P[2][0], P[2][1], P[2][2]);
    g.area = S;
    const double x1 = (P[0][0] + P[1][0]) / 2.0, y1 = (P[0][1] + P[1][1]) / 2.0, z1 = (P[0][2] + P[1][2]) / 2.0;
    const double x2 = (P[1][0] + P[2][0]) / 2.0, y2 = (P[1][1] + P[2][1]) / 2.0, z2 = (P[1][2] + P[2][2]) / 2.0;
    const double x3 = (P[2][0] + P[3][0]) / 2.0, y3 = (P[2][1] + P[3][1]) / 2.0, z3 = (P[2][2] + P[3][2]) / 2.0;
    const double ax = x2 - x1, ay = y2 - y1, az = z2 - z1;
    const double bx = x3 - x1, by = y3 - y1, bz = z3 - z1;
    double n1 = ay * bz - az * by;
    double n2 = az * bx - ax * bz;
    double n3 = ax * by - ay * bx;
    const double nrm = sqrt(n1 * n1 + n2 * n2 + n3 * n3);
    n1 /= nrm;
    n2 /= nrm;
    n3 /= nrm;
    if (n1 * (c0[0] - xc) + n2 * (c0[1] - yc) + n3 * (c0[2] - zc) > 0.0) {
        n1 = -n1;
        n2 = -n2;
        n3 = -n3;
    }
    g.n[0] = n1;
    g.n[1] = n2;
    g.n[2] = n3;
    g.half_dist = 0.0;
    if (c1) {
        const double dx = c0[0] - c1[0], dy = c0[1] - c1[1], dz = c0[2] - c1[2];
        g.half_dist = sqrt(dx * dx + dy * dy + dz * dz) / 2.0;
    }
    return g;
}

__device__ __forceinline__ void load_cc(const double* cc, int nc, int c, double* p) {
    p[0] = cc[c];
    p[1] = cc[nc + c];
    p[2] = cc[2 * nc + c];
}

static __global__ void face_geometry_kernel(MeshView M, Layer L) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= M.nface) return;
    const int nf = M.nface, nn = M.nnode, nc = M.ncell;
    double P[4][3];
#pragma unroll
    for (int k = 0; k < 4; ++k) load_node(L.xyz, nn, M.face_nodes[k * nf + f], P[k]);
    double c0[3], c1[3];
    load_cc(L.cc, nc, M.face_c0[f], c0);
    const int i1 = M.face_c1[f];
    if (i1 >= 0) load_cc(L.cc, nc, i1, c1);
    const FaceGeom g = face_geometry(P, c0, i1 >= 0 ? c1 : nullptr);
    L.fc[f] = g.c[0];
    L.fc[nf + f] = g.c[1];
    L.fc[2 * nf + f] = g.c[2];
    L.fa[f] = g.area;
    L.fn[f] = g.n[0];
    L.fn[nf + f] = g.n[1];
    L.fn[2 * nf + f] = g.n[2];
    L.fd[f] = g.half_dist;
}

// ---------------------------------------------------------------------------
// Reconstruction helpers (first order), Setka_gran_snos.cpp:737-1071.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double polar_angle(double x, double y) {
    if (fabs(x) + fabs(y) < 0.000001) return 0.0;
    if (x < 0) return atan(y / x) + 1.0 * kPi;
    if (x > 0 && y >= 0) return atan(y / x);
    if (x > 0 && y < 0) return atan(y / x) + 2.0 * kPi;
    if (y > 0 && x >= 0 && x <= 0) return kPi / 2.0;
    if (y < 0 && x >= 0 && x <= 0) return 3.0 * kPi / 2.0;
    return 0.0;
}

// Cartesian -> (r, phi, theta) components (Help_funk.cpp:121-135)
__device__ __forceinline__ void to_spherical(double z, double x, double y, double Vz, double Vx, double Vy,
                                             double& Vr, double& Vphi, double& Vtheta) {
    const double r = sqrt(x * x + y * y + z * z);
    const double th = acos(z / r);
    const double ph = polar_angle(x, y);
    const double sth = sin(th), cth = cos(th), sph = sin(ph), cph = cos(ph);
    Vr = Vx * sth * cph + Vy * sth * sph + Vz * cth;
    Vtheta = Vx * cth * cph + Vy * cth * sph - Vz * sth;
    Vphi = -Vx * sph + Vy * cph;
}

// (r, phi, theta) -> Cartesian components (Help_funk.cpp:107-119)
__device__ __forceinline__ void to_cartesian(double z, double x, double y, double Vr, double Vphi, double Vtheta,
                                             double& Vz, double& Vx, double& Vy) {
    const double r = sqrt(x * x + y * y + z * z);
    const double th = acos(z / r);
    const double ph = polar_angle(x, y);
    const double sth = sin(th), cth = cos(th), sph = sin(ph), cph = cos(ph);
    Vx = Vr * sth * cph + Vtheta * cth * cph - Vphi * sph;
    Vy = Vr * sth * sph + Vtheta * cth * sph + Vphi * cph;
    Vz = Vr * cth - Vtheta * sth;
}

// Zone_1 cells are carried radially from the cell centre to the face centre:
// rho, Q, rho_He ~ r^-2, p ~ r^-2gamma, B_r ~ r^-2, B_t ~ r^-1, velocity
// direction rotated (Setka_gran_snos.cpp:744-873).
static __device__ __forceinline__ void zone1_scale(double* s, double ax, double ay, double az, double gx, double gy, double gz,
                                         double gamma) {
    const double r1 = sqrt(ax * ax + ay * ay + az * az);
    const double rr = sqrt(gx * gx + gy * gy + gz * gz);
    const double the1 = acos(gz / rr);
    const bool band = (the1 > kPi / 9 && the1 < 8 * kPi / 9);
#pragma unroll
    for (int ik = 0; ik < 2; ++ik) {
        const int i1 = ik == 0 ? 1 : 5;
        const double X = s[i1], Y = s[i1 + 1], Z = s[i1 + 2];
        double A0, A1, A2;
        if (band)
            to_spherical(az, ax, ay, Z, X, Y, A0, A1, A2);
        else
            to_spherical(ax, ay, az, X, Y, Z, A0, A1, A2);
        if (ik == 1) {
            A0 = A0 * ((r1 / rr) * (r1 / rr));
            A1 = A1 * ((r1) / (rr));
            A2 = A2 * ((r1) / (rr));
        }
        if (band)
            to_cartesian(gz, gx, gy, A0, A1, A2, s[i1 + 2], s[i1], s[i1 + 1]);
        else
            to_cartesian(gx, gy, gz, A0, A1, A2, s[i1], s[i1 + 1], s[i1 + 2]);
    }
    s[0] = s[0] * (r1 * r1) / (rr * rr);
    s[8] = s[8] * (r1 * r1) / (rr * rr);
    s[9] = s[9] * (r1 * r1) / (rr * rr);
    s[4] = s[4] * pow(r1, 2.0 * gamma) / pow(rr, 2.0 * gamma);
}



// Stored flux values per face: rho, m_x, m_y, m_z, E, B_x, B_y, B_z, divB
// (+ Q, rho_He), padded to a 16-byte multiple.
template <typename FT, int NK>
struct FluxLayout {
    static constexpr int n = 9 + NK;
    static constexpr int stride = (sizeof(FT) == 8) ? ((n + 1) & ~1) : ((n + 3) & ~3);
};

}  // namespace titan
#include "tvd.cuh"
namespace titan {

// Second-order neighbours of every face (Setka::Init_TVD,
// Setka_physics.cpp:646-738) on the geometry of layer L: beyond each side, the
// neighbour through another face of that cell whose centre direction from the
// face centre is most opposite to the side's outward normal (the first
// minimum in the cell's face order), dropped when that direction lies within
// acos(0.1) of the face plane. Eigen's dot and normalized() orders.
static __global__ void tvd_neighbours_kernel(MeshView M, Layer L, int* __restrict__ aa, int* __restrict__ bb) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= M.nface) return;
    const int nf = M.nface, nc = M.ncell;
    const double G[3] = {L.fc[f], L.fc[nf + f], L.fc[2 * nf + f]};
    const double nrm[3] = {L.fn[f], L.fn[nf + f], L.fn[2 * nf + f]};
    int pick[2] = {-1, -1};
    for (int side = 0; side < 2; ++side) {
        const int A = side == 0 ? M.face_c0[f] : M.face_c1[f];
        if (A < 0) break;
        double vec[3] = {nrm[0], nrm[1], nrm[2]};
        if (side == 1)
            for (int j = 0; j < 3; ++j) vec[j] = vec[j] * -1.0;
        double best = 2.0;
        for (int k = 0; k < 6; ++k) {
            const int g = M.cell_faces[k * nc + A] & 0x7fffffff;
            if (g == f) continue;
            const int g0 = M.face_c0[g], g1 = M.face_c1[g];
            if (g1 < 0) continue;
            const int cel = g0 == A ? g1 : g0;
            double u[3] = {L.cc[cel] - G[0], L.cc[nc + cel] - G[1], L.cc[2 * nc + cel] - G[2]};
            const double z = (u[0] * u[0] + u[1] * u[1]) + u[2] * u[2];
            if (z > 0.0) {
                const double sz = sqrt(z);
                u[0] = u[0] / sz;
                u[1] = u[1] / sz;
                u[2] = u[2] / sz;
            }
            const double cosine = (vec[0] * u[0] + vec[1] * u[1]) + vec[2] * u[2];
            if (cosine < best) {
                best = cosine;
                pick[side] = cel;
            }
        }
    }
    if (M.face_c1[f] >= 0) {
        for (int side = 0; side < 2; ++side) {
            const int cel = pick[side];
            if (cel < 0) continue;
            double k3[3] = {L.cc[cel] - G[0], L.cc[nc + cel] - G[1], L.cc[2 * nc + cel] - G[2]};
            const double z = (k3[0] * k3[0] + k3[1] * k3[1]) + k3[2] * k3[2];
            if (z > 0.0) {
                const double sz = sqrt(z);
                k3[0] = k3[0] / sz;
                k3[1] = k3[1] / sz;
                k3[2] = k3[2] / sz;
            }
            const double d = (nrm[0] * k3[0] + nrm[1] * k3[1]) + nrm[2] * k3[2];
            if ((side == 0 ? -d : d) < 0.1) pick[side] = -1;
        }
    }
    aa[f] = pick[0];
    bb[f] = pick[1];
}

// Loads through the L2 that the compiler may neither merge with earlier loads
// of the same address nor move: the mixed-precision face kernel reads a face's
// states again after the Riemann solve instead of keeping them live across it.
__device__ __forceinline__ double ld_fresh(const double* p) {
    double v;
    asm volatile("ld.global.cg.f64 %0, [%1];" : "=d"(v) : "l"(p));
    return v;
}

// Face states of one face (Setka::Snos_on_Gran): the two cells' states,
// with the second-order branch (TVD), the Zone_1 radial scaling, the
// Outer_Soft copy with its outflow fix-ups, or the fixed boundary values.
// gc: face centre (set by the caller when MOVE; loaded here otherwise).
// FRESH: every load through ld_fresh (a second evaluation after the solve).
template <int NK, bool MOVE, bool TVD, bool FRESH>
__device__ __forceinline__ void face_states(const FaceArgs& a, int f, int type, int c0, const double* n, double* gc,
                                            double* Ls, double* Rs) {
    const MeshView& M = a.M;
    const Params& P = a.P;
    const int nf = M.nface, nc = M.ncell;
    auto ld = [](const double* p) { return FRESH ? ld_fresh(p) : *p; };
    constexpr int NS = 8 + NK;
#pragma unroll
    for (int k = 0; k < NS; ++k) Ls[k] = ld(a.state + k * nc + c0);
#pragma unroll
    for (int k = NS; k < NV; ++k) Ls[k] = 0.0;
    if (type == 0) {
        const int c1 = M.face_c1[f];
#pragma unroll
        for (int k = 0; k < NS; ++k) Rs[k] = ld(a.state + k * nc + c1);
#pragma unroll
        for (int k = NS; k < NV; ++k) Rs[k] = 0.0;
        bool second = false;
        if (TVD) {
            const int aa = M.face_aa[f], bb = M.face_bb[f];
            if (aa >= 0 && bb >= 0 && M.cell_tvd[c0] && M.cell_tvd[c1] && (M.face_surf[f] != 2 || P.snos_on_hp)) {
                // second-order branch (Setka_gran_snos.cpp:188-735)
                if (!MOVE) {
                    gc[0] = ld(a.L1.fc + f);
                    gc[1] = ld(a.L1.fc + nf + f);
                    gc[2] = ld(a.L1.fc + 2 * nf + f);
                }
                const int c4[4] = {aa, c0, c1, bb};
                double S4[4][NV], X4[4][3];
                int t4[4];
#pragma unroll
                for (int i = 0; i < 4; ++i) {
#pragma unroll
                    for (int k = 0; k < NS; ++k) S4[i][k] = ld(a.state + k * nc + c4[i]);
#pragma unroll
                    for (int k = NS; k < NV; ++k) S4[i][k] = 0.0;
#pragma unroll
                    for (int k = 0; k < 3; ++k) X4[i][k] = ld(a.L1.cc + k * nc + c4[i]);
                    t4[i] = M.cell_type[c4[i]];
                }
                snos_tvd<NK>(S4, X4, t4, gc, P.gamma, Ls, Rs);
                second = true;
            }
        }
        const bool z0 = !second && M.cell_type[c0] == 1, z1 = !second && M.cell_type[c1] == 1;
        if (z0 || z1) {
            if (!MOVE) {
                gc[0] = ld(a.L1.fc + f);
                gc[1] = ld(a.L1.fc + nf + f);
                gc[2] = ld(a.L1.fc + 2 * nf + f);
            }
            if (z0)
                zone1_scale(Ls, ld(a.L1.cc + c0), ld(a.L1.cc + nc + c0), ld(a.L1.cc + 2 * nc + c0), gc[0], gc[1],
                            gc[2], P.gamma);
            if (z1)
                zone1_scale(Rs, ld(a.L1.cc + c1), ld(a.L1.cc + nc + c1), ld(a.L1.cc + 2 * nc + c1), gc[0], gc[1],
                            gc[2], P.gamma);
        }
    } else if (type == 3) {
        // Outer_Soft: copy the interior cell, with the reference's outflow fix-ups
        if (P.soft_fixups) {
            if (n[0] < -0.95) {
                if (Ls[1] > P.velosity_inf / 7.0) Ls[1] = P.velosity_inf / 5.0;
            } else if (Ls[1] * n[0] + Ls[2] * n[1] + Ls[3] * n[2] < 0.0) {
                Ls[1] = 0.1 * n[0];
                Ls[2] = 0.1 * n[1];
                Ls[3] = 0.1 * n[2];
            }
        }
#pragma unroll
        for (int k = 0; k < NV; ++k) Rs[k] = Ls[k];
    } else {
        // Inner_Hard / Outer_Hard: fixed face values
        const int row = M.face_bc[f];
#pragma unroll
        for (int k = 0; k < NV; ++k) Rs[k] = ld(M.bc_vals + k * M.nbc + row);
    }
}

template <typename R, typename FT, int NK, bool MOVE, int BS, int MINB, bool TVD = false>
__global__ void __launch_bounds__(BS, MINB) face_flux_kernel(FaceArgs a) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    double contrib = 100000000.0;  // identity of the min (Setka_physics.cpp:1607)
    if (f < a.M.nface && a.st->err_kind == 0) {
        const MeshView& M = a.M;
        const Params& P = a.P;
        const int nf = M.nface, nc = M.ncell;
        const int type = M.face_type[f];
        const int c0 = M.face_c0[f];
        double n[3], area, dist = 0.0, gc[3];
        double w = 0.0;
        if (MOVE) {
            // geometry of this layer from the face's nodes (as Gran::Culc_measure),
            // then the face speed from the node displacement (Gran::culc_velosity)
            const int nn = M.nnode;
            int nid[4];
            double P[4][3], Q[4][3];
            // both layers' nodes in one batch of loads, ahead of the arithmetic
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                nid[k] = M.face_nodes[k * nf + f];
                load_node(a.L1.xyz, nn, nid[k], P[k]);
                load_node(a.xyz2, nn, nid[k], Q[k]);
            }
            double cA[3], cB[3];
            load_cc(a.L1.cc, nc, c0, cA);
            if (type == 0) load_cc(a.L1.cc, nc, M.face_c1[f], cB);
            const FaceGeom g = face_geometry(P, cA, type == 0 ? cB : nullptr);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                n[k] = g.n[k];
                gc[k] = g.c[k];
            }
            area = g.area;
            dist = g.half_dist;
            const double time = a.st->dt;
            double ddot = 0.0;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const double dx = Q[k][0] - P[k][0];
                const double dy = Q[k][1] - P[k][1];
                const double dz = Q[k][2] - P[k][2];
                ddot = ddot + (dx * n[0] + dy * n[1] + dz * n[2]);
            }
            w = ddot / 4.0 / time;
        } else {
            n[0] = a.L1.fn[f];
            n[1] = a.L1.fn[nf + f];
            n[2] = a.L1.fn[2 * nf + f];
            area = a.L1.fa[f];
        }
        double Ls[NV], Rs[NV];
        face_states<NK, MOVE, TVD, false>(a, f, type, c0, n, gc, Ls, Rs);
        int method;
        if (P.method_policy == 1) {
            const double bb = ((Ls[5] * Ls[5] + Ls[6] * Ls[6] + Ls[7] * Ls[7]) +
                               (Rs[5] * Rs[5] + Rs[6] * Rs[6] + Rs[7] * Rs[7])) / 2.0;
            const double pp = (Ls[4] + Rs[4]) / 2.0;
            method = (bb / (4.0 * kPi) / (2.0 * pp) > P.beta_switch) ? 3 : 2;
        } else {
            method = M.face_method[f];
        }
        // Powell term: the face-normal B of the two states, averaged (divB * area)
        const double bsum = 0.5 * (n[0] * (Ls[5] + Rs[5]) + n[1] * (Ls[6] + Rs[6]) + n[2] * (Ls[7] + Rs[7]));
        const int surf = M.face_surf[f];
        RiemannFlags fl;
        fl.null_bn = false;
        fl.n_disc = 0;
        fl.left_ydar = (surf == 1 && P.TS_hard);
        fl.contact = (surf == 2 && P.contact_hard);
        double qd[8], kqd[NK > 0 ? NK : 1], dsl_d, dsr_d, bsum_f = bsum;
        if (P.bn_in_p_on_hp && surf == 2) {
            // HP face with the magnetic pressure in p: the exact gas-dynamic
            // solver (Setka_physics.cpp:2378-2409); no B or passive flux, no PdivB
            const GodunovFlux gd =
                godunov_hp_face(n[0], n[1], n[2], w, Ls[0], Ls[1], Ls[2], Ls[3], Ls[4], Ls[5], Ls[6], Ls[7], Rs[0],
                                Rs[1], Rs[2], Rs[3], Rs[4], Rs[5], Rs[6], Rs[7], P.contact_hard, P.gamma);
            if (gd.rc) record_error(a.st, 14 + gd.rc, f);
#pragma unroll
            for (int k = 0; k < 5; ++k) qd[k] = gd.q[k];
            qd[5] = qd[6] = qd[7] = 0.0;
#pragma unroll
            for (int k = 0; k < NK; ++k) kqd[k] = 0.0;
            dsl_d = gd.dsl;
            dsr_d = gd.dsr;
            bsum_f = 0.0;
        } else {
        R qL[8], qR[8], kl[NK > 0 ? NK : 1], kr[NK > 0 ? NK : 1], q[8], kq[NK > 0 ? NK : 1], nr[3];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            qL[k] = R(Ls[k]);
            qR[k] = R(Rs[k]);
        }
#pragma unroll
        for (int k = 0; k < NK; ++k) {
            kl[k] = R(Ls[8 + k]);
            kr[k] = R(Rs[8 + k]);
        }
        nr[0] = R(n[0]);
        nr[1] = R(n[1]);
        nr[2] = R(n[2]);
        R dsl, dsc, dsr;
        // mixed precision: the FP32 solver reports faces that lie wholly in one
        // side's region, whose flux is then formed again in FP64
        constexpr bool kMixed = sizeof(R) < sizeof(double);
        int upw = 0;
        R wvo = R(0);
        const int rc = riemann_flux<R, NK, kMixed>(method, nr, R(w), qL, qR, kl, kr, q, kq, dsl, dsc, dsr, fl,
                                                    R(P.gamma), &upw, &wvo);
        if (rc) record_error(a.st, 10 + rc, f);
#pragma unroll
        for (int k = 0; k < 8; ++k) qd[k] = double(q[k]);
#pragma unroll
        for (int k = 0; k < NK; ++k) kqd[k] = double(kq[k]);
        if (kMixed && upw) {
            // the face's states again, loaded anew rather than kept live across the solve
            double L2[NV], R2[NV];
            face_states<NK, MOVE, TVD, true>(a, f, type, c0, n, gc, L2, R2);
            upwind_flux_fp64<NK>(n, double(wvo), L2, R2, L2 + 8, R2 + 8, upw == 1, double(dsl), double(dsr),
                                 fl.null_bn, P.gamma, qd, kqd);
        }
        dsl_d = double(dsl);
        dsr_d = double(dsr);
        }
        if (type == 0 && !(M.face_nodt && M.face_nodt[f])) {
            if (!MOVE) dist = a.L1.fd[f];
            const double dnt = P.KFL * dist / (rmax(fabs(dsl_d), fabs(dsr_d)) + fabs(w));
            contrib = 10000000.0;
            if (dnt < contrib) contrib = dnt;
        } else {
            contrib = 10000000.0;
        }
        using L = FluxLayout<FT, NK>;
        FT out[L::stride];
#pragma unroll
        for (int k = 0; k < 8; ++k) out[k] = FT(qd[k] * area);
        out[8] = FT(bsum_f * area);
#pragma unroll
        for (int k = 0; k < NK; ++k) out[9 + k] = FT(kqd[k] * area);
#pragma unroll
        for (int k = L::n; k < L::stride; ++k) out[k] = FT(0);
        FT* dst = reinterpret_cast<FT*>(a.flux) + size_t(f) * L::stride;
        if (sizeof(FT) == 8) {
#pragma unroll
            for (int k = 0; k < L::stride; k += 2)
                reinterpret_cast<double2*>(dst)[k / 2] = make_double2(double(out[k]), double(out[k + 1]));
        } else {
#pragma unroll
            for (int k = 0; k < L::stride; k += 4)
                reinterpret_cast<float4*>(dst)[k / 4] =
                    make_float4(float(out[k]), float(out[k + 1]), float(out[k + 2]), float(out[k + 3]));
        }
    }
    // CFL minimum: warp shuffle, then shared memory across the block, then one
    // atomicMin on the ordered bit pattern (all candidates are >= 0).
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) contrib = fmin(contrib, __shfl_xor_sync(0xffffffffu, contrib, o));
    __shared__ double red[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) red[wid] = contrib;
    __syncthreads();
    if (wid == 0) {
        double v = (lane < (int)(blockDim.x >> 5)) ? red[lane] : 100000000.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (lane == 0 && v < 100000000.0)
            atomicMin(&a.st->dt_next_bits, (unsigned long long)__double_as_longlong(v));
    }
}



// Bera charge-exchange sources of the plasma (Setka_physics.cpp:766-1258,
// no pickup ions), returning m_x, m_y, m_z, E times n_H_LISM / Kn.
static __device__ __forceinline__ void bera_sources(const Params& P, const double* prim, int ctype, const double* H, int nc,
                                          int c, double* S) {
    const double rho = prim[0], p = prim[4], Q = prim[8], rho_He = prim[9];
    int zone;
    if (Q / rho < 50.0)
        zone = (ctype == 1) ? 1 : 2;
    else
        zone = (ctype == 4) ? 4 : 3;
    const int al = (zone - 1 <= 2) ? 2 : 1;  // Plasma_components_1 receives zone - 1
    double rho_p = -(kMeDmp * al * rho_He + 4.0 * (-rho + rho_He)) / (4.0 * (1.0 + kMeDmp));
    double T_p = 8.0 * (1.0 + kMeDmp) * p / (8.0 * rho - (7.0 - al + (-1.0 + al) * kMeDmp) * rho_He);
    if (rho_p <= 1e-8) rho_p = 1e-8;
    if (T_p <= 1e-8) T_p = 1e-8;
    if (T_p > 1e5) T_p = 1e5;
    const double Vp0 = prim[1], Vp1 = prim[2], Vp2 = prim[3];
    double mxs = 0.0, mys = 0.0, mzs = 0.0, Es = 0.0;
    for (int h = 0; h < P.nh; ++h) {
        const double rho_h = H[(5 * h + 0) * nc + c];
        const double Vh0 = H[(5 * h + 1) * nc + c], Vh1 = H[(5 * h + 2) * nc + c], Vh2 = H[(5 * h + 3) * nc + c];
        const double T_h = 2.0 * H[(5 * h + 4) * nc + c] / rmax(rho_h, 1e-9);
        const double d0 = Vp0 - Vh0, d1 = Vp1 - Vh1, d2 = Vp2 - Vh2;
        const double uu = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
        const double U_ph = sqrt((4.0 / kPi) * (T_p + T_h) + uu * uu);
        const double U_hp = sqrt((4.0 / kPi) * (T_h + T_p) + uu * uu);
        const double Um_ph = sqrt((16.0 / kPi) * T_p + (9.0 * kPi / 4.0) * T_h + 4.0 * (uu * uu));
        const double Um_hp = sqrt((16.0 / kPi) * T_h + (9.0 * kPi / 4.0) * T_p + 4.0 * (uu * uu));
        const double UE_ph = sqrt((4.0 / kPi) * T_p + (64.0 / 9.0 / kPi) * T_h + uu * uu);
        const double UE_hp = sqrt((4.0 / kPi) * T_h + (64.0 / 9.0 / kPi) * T_p + uu * uu);
        const double a_ph = 1.0 - P.par_a_2 * log(U_ph);
        const double a_hp = 1.0 - P.par_a_2 * log(U_hp);
        const double k_hp = (a_hp * a_hp) * rho_p * rho_h;
        const double k_ph = (a_ph * a_ph) * rho_p * rho_h;
        const double t_hp = T_p / Um_hp, t_ph = T_h / Um_ph;
        const double Hm_hp0 = k_hp * (U_hp * Vp0 + t_hp * d0);
        const double Hm_hp1 = k_hp * (U_hp * Vp1 + t_hp * d1);
        const double Hm_hp2 = k_hp * (U_hp * Vp2 + t_hp * d2);
        const double Hm_ph0 = k_ph * (U_ph * Vh0 - t_ph * d0);
        const double Hm_ph1 = k_ph * (U_ph * Vh1 - t_ph * d1);
        const double Hm_ph2 = k_ph * (U_ph * Vh2 - t_ph * d2);
        const double vp2 = Vp0 * Vp0 + Vp1 * Vp1 + Vp2 * Vp2;
        const double vh2 = Vh0 * Vh0 + Vh1 * Vh1 + Vh2 * Vh2;
        const double vpd = Vp0 * d0 + Vp1 * d1 + Vp2 * d2;
        const double vhd = Vh0 * d0 + Vh1 * d1 + Vh2 * d2;
        const double HE_hp = k_hp * (0.5 * U_hp * vp2 + t_hp * vpd + 3.0 / 4.0 * T_p * UE_hp);
        const double HE_ph = k_ph * (0.5 * U_ph * vh2 - t_ph * vhd + 3.0 / 4.0 * T_h * UE_ph);
        mxs += (-Hm_hp0 + Hm_ph0);
        mys += (-Hm_hp1 + Hm_ph1);
        mzs += (-Hm_hp2 + Hm_ph2);
        Es += (-HE_hp + HE_ph);
    }
    const double ddp = (P.par_n_H_LISM / P.par_Kn);
    S[0] = mxs * ddp;
    S[1] = mys * ddp;
    S[2] = mzs * ddp;
    S[3] = Es * ddp;
}


// ---------------------------------------------------------------------------
// Permutation kernels for upload/download (SoA fields of length n).
// dst[k][i] = src[k][perm[i]]  (gather)   /   dst[k][perm[i]] = src[k][i] (scatter)
// ---------------------------------------------------------------------------
static __global__ void gather_fields_kernel(const double* __restrict__ src, double* __restrict__ dst,
                                     const int* __restrict__ perm, int n, int nfields) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int j = perm[i];
    for (int k = 0; k < nfields; ++k) dst[size_t(k) * n + i] = src[size_t(k) * n + j];
}

static __global__ void scatter_fields_kernel(const double* __restrict__ src, double* __restrict__ dst,
                                      const int* __restrict__ perm, int n, int nfields) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int j = perm[i];
    for (int k = 0; k < nfields; ++k) dst[size_t(k) * n + j] = src[size_t(k) * n + i];
}

// Stateless batched Riemann solver (parity checks against the reference
// solver and FP32 error measurements). AoS inputs, as the reference's qqq.
template <typename R>
__global__ void riemann_batch_kernel(long long n, const signed char* __restrict__ ns, const double* __restrict__ nrm,
                                     const double* __restrict__ w, const double* __restrict__ q1,
                                     const double* __restrict__ q2, double* __restrict__ flux,
                                     double* __restrict__ ds, int* __restrict__ rc, int flags, double gamma) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    R a[8], b[8], q[8], nr[3], dummy[1], ko[1];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        a[k] = R(q1[8 * i + k]);
        b[k] = R(q2[8 * i + k]);
    }
    nr[0] = R(nrm[3 * i]);
    nr[1] = R(nrm[3 * i + 1]);
    nr[2] = R(nrm[3 * i + 2]);
    RiemannFlags fl;
    fl.null_bn = (flags & 1) != 0;
    fl.left_ydar = (flags & 2) != 0;
    fl.contact = (flags & 4) != 0;
    fl.n_disc = (flags >> 4) & 3;
    R dsl, dsc, dsr;
    rc[i] = riemann_flux<R, 0>(ns[i], nr, R(w[i]), a, b, dummy, dummy, q, ko, dsl, dsc, dsr, fl, R(gamma));
#pragma unroll
    for (int k = 0; k < 8; ++k) flux[8 * i + k] = double(q[k]);
    ds[3 * i] = double(dsl);
    ds[3 * i + 1] = double(dsc);
    ds[3 * i + 2] = double(dsr);
}

}  // namespace titan
