// Second-order (TVD) face reconstruction of the plasma step, restating
// Setka::Snos_on_Gran's second-order branch (TITAN/source/Setka_gran_snos.cpp:
// 188-735) with the helpers minmod / linear / linear2 (Help_funk.cpp:43-70).
//
// Cells on the line AA - A -|- B - BB (AA beyond cells[0], BB beyond
// cells[1], chosen once by Setka::Init_TVD, Setka_physics.cpp:646-738) sit at
// coordinates -dd1-d1, -d1, 0 (the face centre), d2, d2+dd2. `linear` is the
// minmod of the two slopes through the middle point, `linear2` the line
// through two points, both evaluated at the face. The branch taken depends on
// the zone types of the four cells: all-Zone_1 lines carry the vector fields
// in spherical components and scale rho, Q, rho_He by r^2 and p by r^(2 gamma)
// (B_r by r^2, B_phi and B_theta by r); the Zone_1 / Zone_2 transitions and
// the Zone_2/3/4 transitions switch sides to one-sided lines. On the
// transition branches the reference's `if` / `if ... else` sequence
// (Setka_gran_snos.cpp:502-532, :617-644) overwrites the r^2 scaling of
// rho, Q and rho_He with the plain line, so only p stays scaled there; that
// is reproduced. Every expression keeps the reference's order (the FP64
// translation unit is built without contraction).
#pragma once

#include "step_types.h"

namespace titan {

__device__ __forceinline__ int tvd_signum(double x) {
    return x > 0.00000001 ? 1 : (x < -0.00000001 ? -1 : 0);
}

__device__ __forceinline__ double tvd_minmod(double x, double y) {
    const int s = tvd_signum(x) + tvd_signum(y);
    if (s == 0) return 0.0;
    const double ax = fabs(x), ay = fabs(y);
    return (s / 2.0) * ((ay < ax) ? ay : ax);
}

// linear(x1, t1, x2, t2, x3, t3, 0)
__device__ __forceinline__ double tvd_lin3(double x1, double t1, double x2, double t2, double x3, double t3) {
    const double y = 0.0;
    const double d = tvd_minmod((t1 - t2) / (x1 - x2), (t2 - t3) / (x2 - x3));
    return (d * (y - x2) + t2);
}

// linear2(x1, t1, x2, t2, 0)
__device__ __forceinline__ double tvd_lin2(double x1, double t1, double x2, double t2) {
    const double y = 0.0;
    const double d = (t1 - t2) / (x1 - x2);
    return (d * (y - x2) + t2);
}

__device__ __forceinline__ double tvd_norm3(double x, double y, double z) { return sqrt(x * x + y * y + z * z); }

// Spherical components (Vr, Vphi, Vtheta) of the vector (vx, vy, vz) at X, in
// the frame the face's band test selects; and back to Cartesian at G.
__device__ __forceinline__ void tvd_sph(bool band, const double* X, double vx, double vy, double vz, double* o) {
    if (band)
        to_spherical(X[2], X[0], X[1], vz, vx, vy, o[0], o[1], o[2]);
    else
        to_spherical(X[0], X[1], X[2], vx, vy, vz, o[0], o[1], o[2]);
}

__device__ __forceinline__ void tvd_cart(bool band, const double* G, const double* Vs, double* side, int k0) {
    if (band)
        to_cartesian(G[2], G[0], G[1], Vs[0], Vs[1], Vs[2], side[k0 + 2], side[k0], side[k0 + 1]);
    else
        to_cartesian(G[0], G[1], G[2], Vs[0], Vs[1], Vs[2], side[k0], side[k0 + 1], side[k0 + 2]);
}

// Face states L, R (NV each; rows >= 8 + NK are not read) of an interior
// face on the second-order branch. S[i][k]: state k of cell i (AA, A, B, BB);
// X[i]: centres; ct[i]: Type_cell; G: face centre.
template <int NK>
__device__ __forceinline__ void snos_tvd(const double (*S)[NV], const double (*X)[3], const int* ct, const double* G,
                                         double gamma, double* L, double* R) {
    double v0 = X[1][0] - G[0], v1 = X[1][1] - G[1], v2 = X[1][2] - G[2];
    const double d1 = tvd_norm3(v0, v1, v2);
    v0 = X[2][0] - G[0];
    v1 = X[2][1] - G[1];
    v2 = X[2][2] - G[2];
    const double d2 = tvd_norm3(v0, v1, v2);
    v0 = X[1][0] - X[0][0];
    v1 = X[1][1] - X[0][1];
    v2 = X[1][2] - X[0][2];
    const double dd1 = tvd_norm3(v0, v1, v2);
    v0 = X[2][0] - X[3][0];
    v1 = X[2][1] - X[3][1];
    v2 = X[2][2] - X[3][2];
    const double dd2 = tvd_norm3(v0, v1, v2);
    const double xAA = -dd1 - d1, xA = -d1, xB = d2, xBB = d2 + dd2;
    const int a0 = ct[0], a1 = ct[1], b1 = ct[2], b0 = ct[3];
    const bool z1111 = a0 == 1 && a1 == 1 && b1 == 1 && b0 == 1;
    const bool z1112 = a0 == 1 && a1 == 1 && b1 == 1 && b0 == 2;
    const bool z1122 = a0 == 1 && a1 == 1 && b1 == 2 && b0 == 2;
    const bool z1222 = a0 == 1 && a1 == 2 && b1 == 2 && b0 == 2;
    if (z1111 || z1112 || z1122) {
        const double r3 = tvd_norm3(X[0][0], X[0][1], X[0][2]), r1 = tvd_norm3(X[1][0], X[1][1], X[1][2]);
        const double rr = tvd_norm3(G[0], G[1], G[2]);
        const double r2 = tvd_norm3(X[2][0], X[2][1], X[2][2]), r4 = tvd_norm3(X[3][0], X[3][1], X[3][2]);
        const double the1 = acos(G[2] / rr);
        const bool band = the1 > kPi / 9 && the1 < 8 * kPi / 9;
#pragma unroll 1
        for (int ik = 0; ik < 2; ++ik) {
            const int k0 = ik == 0 ? 1 : 5;
            double VAA[3], VA[3], VB[3], VBB[3], Vl[3], Vr[3];
            tvd_sph(band, X[0], S[0][k0], S[0][k0 + 1], S[0][k0 + 2], VAA);
            tvd_sph(band, X[1], S[1][k0], S[1][k0 + 1], S[1][k0 + 2], VA);
            if (z1111) {
                tvd_sph(band, X[2], S[2][k0], S[2][k0 + 1], S[2][k0 + 2], VB);
                tvd_sph(band, X[3], S[3][k0], S[3][k0 + 1], S[3][k0 + 2], VBB);
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    if (ik == 1) {
                        if (i == 0) {
                            Vl[i] = tvd_lin3(xAA, VAA[i] * ((r3) * (r3)), xA, VA[i] * ((r1) * (r1)), xB,
                                             VB[i] * ((r2) * (r2))) / ((rr) * (rr));
                            Vr[i] = tvd_lin3(xA, VA[i] * ((r1) * (r1)), xB, VB[i] * ((r2) * (r2)), xBB,
                                             VBB[i] * ((r4) * (r4))) / ((rr) * (rr));
                        } else {
                            Vl[i] = tvd_lin3(xAA, VAA[i] * (r3), xA, VA[i] * (r1), xB, VB[i] * (r2)) / (rr);
                            Vr[i] = tvd_lin3(xA, VA[i] * (r1), xB, VB[i] * (r2), xBB, VBB[i] * (r4)) / (rr);
                        }
                    } else {
                        Vl[i] = tvd_lin3(xAA, VAA[i], xA, VA[i], xB, VB[i]);
                        Vr[i] = tvd_lin3(xA, VA[i], xB, VB[i], xBB, VBB[i]);
                    }
                }
                tvd_cart(band, G, Vl, L, k0);
                tvd_cart(band, G, Vr, R, k0);
            } else if (z1112) {
                tvd_sph(band, X[2], S[2][k0], S[2][k0 + 1], S[2][k0 + 2], VB);
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    Vl[i] = tvd_lin3(xAA, VAA[i], xA, VA[i], xB, VB[i]);
                    Vr[i] = tvd_lin2(xA, VA[i], xB, VB[i]);
                }
                tvd_cart(band, G, Vl, L, k0);
                tvd_cart(band, G, Vr, R, k0);
            } else {
#pragma unroll
                for (int i = 0; i < 3; ++i) Vl[i] = tvd_lin2(xAA, VAA[i], xA, VA[i]);
                tvd_cart(band, G, Vl, L, k0);
            }
        }
        const double g2 = 2.0 * gamma;
        const double p3 = pow(r3, g2), p1 = pow(r1, g2), p2 = pow(r2, g2), p4 = pow(r4, g2), pr = pow(rr, g2);
        // p (r^(2 gamma))
        if (z1111) {
            L[4] = tvd_lin3(xAA, S[0][4] * p3, xA, S[1][4] * p1, xB, S[2][4] * p2) / pr;
            R[4] = tvd_lin3(xA, S[1][4] * p1, xB, S[2][4] * p2, xBB, S[3][4] * p4) / pr;
        } else if (z1112) {
            L[4] = tvd_lin3(xAA, S[0][4] * p3, xA, S[1][4] * p1, xB, S[2][4] * p2) / pr;
            R[4] = tvd_lin2(xA, S[1][4] * p1, xB, S[2][4] * p2) / pr;
        } else {
            L[4] = tvd_lin2(xAA, S[0][4] * p3, xA, S[1][4] * p1) / pr;
            R[4] = tvd_lin2(xB, S[2][4], xBB, S[3][4]);
        }
        // rho, Q, rho_He (r^2 on the all-Zone_1 branch only)
#pragma unroll
        for (int q = 0; q < 1 + NK; ++q) {
            const int k = q == 0 ? 0 : 7 + q;
            if (z1111) {
                L[k] = tvd_lin3(xAA, S[0][k] * ((r3) * (r3)), xA, S[1][k] * ((r1) * (r1)), xB,
                                S[2][k] * ((r2) * (r2))) / ((rr) * (rr));
                R[k] = tvd_lin3(xA, S[1][k] * ((r1) * (r1)), xB, S[2][k] * ((r2) * (r2)), xBB,
                                S[3][k] * ((r4) * (r4))) / ((rr) * (rr));
            } else if (z1112) {
                L[k] = tvd_lin3(xAA, S[0][k], xA, S[1][k], xB, S[2][k]);
                R[k] = tvd_lin2(xA, S[1][k], xB, S[2][k]);
            } else {
                L[k] = tvd_lin2(xAA, S[0][k], xA, S[1][k]);
                R[k] = tvd_lin2(xB, S[2][k], xBB, S[3][k]);
            }
        }
        if (z1122) {
#pragma unroll
            for (int k = 1; k < 8; ++k)
                if (k != 4) R[k] = tvd_lin2(xB, S[2][k], xBB, S[3][k]);
        }
    } else {
        const bool l2 = (a0 == 2 && a1 == 2 && b1 == 3 && b0 == 3) || (a0 == 3 && a1 == 3 && b1 == 4 && b0 == 4);
        const bool l3 = (a0 == 2 && a1 == 2 && b1 == 2 && b0 == 3) || (a0 == 3 && a1 == 3 && b1 == 3 && b0 == 4);
        const bool l4 =
            z1222 || (a0 == 2 && a1 == 3 && b1 == 3 && b0 == 3) || (a0 == 3 && a1 == 4 && b1 == 4 && b0 == 4);
#pragma unroll
        for (int k = 0; k < 8 + NK; ++k) {
            if (l2) {
                L[k] = tvd_lin2(xAA, S[0][k], xA, S[1][k]);
                R[k] = tvd_lin2(xB, S[2][k], xBB, S[3][k]);
            } else if (l3) {
                L[k] = tvd_lin3(xAA, S[0][k], xA, S[1][k], xB, S[2][k]);
                R[k] = tvd_lin2(xA, S[1][k], xB, S[2][k]);
            } else if (l4) {
                L[k] = tvd_lin2(xA, S[1][k], xB, S[2][k]);
                R[k] = tvd_lin3(xA, S[1][k], xB, S[2][k], xBB, S[3][k]);
            } else {
                L[k] = tvd_lin3(xAA, S[0][k], xA, S[1][k], xB, S[2][k]);
                R[k] = tvd_lin3(xA, S[1][k], xB, S[2][k], xBB, S[3][k]);
            }
        }
    }
    // positivity fall-back to the cell value (Setka_gran_snos.cpp:710-720)
    if (L[0] < 0.0000001) L[0] = S[1][0];
    if (L[4] < 0.0000001) L[4] = S[1][4];
    if (R[0] < 0.0000001) R[0] = S[2][0];
    if (R[4] < 0.0000001) R[4] = S[2][4];
#pragma unroll
    for (int k = 8; k < 8 + NK; ++k) {
        if (L[k] < 0.0000001) L[k] = S[1][k];
        if (R[k] < 0.0000001) R[k] = S[2][k];
    }
}

}  // namespace titan
