// Device-side MHD Riemann solvers for one moving face.
//
// Computes what TITAN's Phys_param::chlld (TITAN/source/Phys_param.cpp:882-1878)
// computes: the Lax (n_state 0), HLL (1), HLLC (2) and HLLD (3) fluxes in the
// frame of a face moving with normal speed w, rotated into the face basis of
// get_bazis (TITAN/source/Help_funk.cpp:219-232), with the Powell-form normal
// B flux -SN*(bR-bL) - w*bn and the sqrt(4*pi) Gaussian rescale of B.
//
// Every value is written with the reference's expression tree, so that in
// double precision, compiled without FMA contraction (the FP64 translation
// unit uses -fmad=false), it rounds exactly as the reference's x86-64 build.
// The evaluation ORDER differs where that saves work on the GPU: the HLLC and
// HLLD wave region ("zone") is decided first from the wave speeds, replaying
// the reference's sequence of tests (including the HLLD zone-5 overwrite at
// ties and when |bn| <= epsb), and only the star states that region needs are
// formed; the averaged-state speed is formed only for the estimates that use
// it. The single precision instantiation runs the same algorithm in float.
#pragma once
#ifdef __CUDACC__
#include <cuda_runtime.h>
#endif
#include <math.h>

namespace titan {

template <typename R>
struct RConst;
template <>
struct RConst<double> {
    // sqrt(4*pi) rounded to double, the value TITAN/source/Header.h:99 computes
    static __device__ __forceinline__ double spi4() { return 3.5449077018110318; }
    static __device__ __forceinline__ double epsb() { return 1E-4; }
    static __device__ __forceinline__ double tt_eps() { return 0.000000001; }
};
template <>
struct RConst<float> {
    static __device__ __forceinline__ float spi4() { return 3.5449077018110318f; }
    static __device__ __forceinline__ float epsb() { return 1E-4f; }
    static __device__ __forceinline__ float tt_eps() { return 0.000000001f; }
};

// std::min / std::max argument semantics (the reference uses <algorithm>)
template <typename R>
__device__ __forceinline__ R rmin(R a, R b) { return (b < a) ? b : a; }
template <typename R>
__device__ __forceinline__ R rmax(R a, R b) { return (a < b) ? b : a; }

// Orthonormal (t, m) completing the unit normal n.
template <typename R>
__device__ __forceinline__ void face_basis(const R n[3], R t[3], R m[3]) {
    R a0 = R(1), a1 = R(0), a2 = R(0);
    if (fabs(n[0] * a0 + n[1] * a1 + n[2] * a2) > R(0.9)) {
        a0 = R(0);
        a1 = R(1);
    }
    const R c0 = a1 * n[2] - a2 * n[1];
    const R c1 = a2 * n[0] - a0 * n[2];
    const R c2 = a0 * n[1] - a1 * n[0];
    const R z = c0 * c0 + c1 * c1 + c2 * c2;
    if (z > R(0)) {
        const R s = sqrt(z);
        t[0] = c0 / s;
        t[1] = c1 / s;
        t[2] = c2 / s;
    } else {
        t[0] = c0;
        t[1] = c1;
        t[2] = c2;
    }
    m[0] = n[1] * t[2] - n[2] * t[1];
    m[1] = n[2] * t[0] - n[0] * t[2];
    m[2] = n[0] * t[1] - n[1] * t[0];
}

struct RiemannFlags {
    bool null_bn;
    bool left_ydar;
    bool contact;
    int n_disc;
};

// Flux F and conserved vector U of one side in the face frame.
template <typename R>
__device__ __forceinline__ void side_flux(R r, const R v[3], const R b[3], R pt, R e, R sbv, R F[8], R U[8]) {
    F[0] = r * v[0];
    F[1] = r * v[0] * v[0] + pt - b[0] * b[0];
    F[2] = r * v[0] * v[1] - b[0] * b[1];
    F[3] = r * v[0] * v[2] - b[0] * b[2];
    F[4] = (e + pt) * v[0] - b[0] * sbv;
    F[5] = R(0);
    F[6] = v[0] * b[1] - v[1] * b[0];
    F[7] = v[0] * b[2] - v[2] * b[0];
    U[0] = r;
    U[1] = r * v[0];
    U[2] = r * v[1];
    U[3] = r * v[2];
    U[4] = e;
    U[5] = b[0];
    U[6] = b[1];
    U[7] = b[2];
}

// Returns 0 on success; 1/2/3 where the reference would abort (no admissible
// wave region, i.e. NaN speeds) for the HLL/HLLC/HLLD branches, 4 for a bad
// n_state. q1/q2: rho, u, v, w, p, Bx, By, Bz (Gaussian B). qout: 8 fluxes.
// kl/kr/kout: NK passive scalars carried by the contact.
// TRACK: when the face lies wholly in one side's region (HLLC zones 1/4, HLLD
// zones 1/6), *upw is set to 1 (left) or 2 (right) and *wv_out to the frame
// speed used, so that a caller can form that flux again in higher precision
// (upwind_flux_fp64); qout is filled as usual either way.
template <typename R, int NK, bool TRACK = false>
__device__ __forceinline__ int riemann_flux(int n_state, const R nrm[3], R w, const R* q1, const R* q2,
                                            const R* kl, const R* kr, R* qout, R* kout, R& dsl, R& dsc,
                                            R& dsr, RiemannFlags fl, R gamma, int* upw = nullptr,
                                            R* wv_out = nullptr) {
    const R spi4 = RConst<R>::spi4();
    const R g1 = gamma - R(1);
    R wv = w;
    const R r1 = q1[0], u1 = q1[1], v1 = q1[2], w1 = q1[3], p1 = q1[4];
    const R bx1 = q1[5] / spi4, by1 = q1[6] / spi4, bz1 = q1[7] / spi4;
    const R r2 = q2[0], u2 = q2[1], v2 = q2[2], w2 = q2[3], p2 = q2[4];
    const R bx2 = q2[5] / spi4, by2 = q2[6] / spi4, bz2 = q2[7] / spi4;

    R n[3] = {nrm[0], nrm[1], nrm[2]}, t[3], m[3];
    face_basis(n, t, m);

    R vL[3], vR[3], bL[3], bR[3];
    vL[0] = n[0] * u1 + n[1] * v1 + n[2] * w1;
    vL[1] = t[0] * u1 + t[1] * v1 + t[2] * w1;
    vL[2] = m[0] * u1 + m[1] * v1 + m[2] * w1;
    vR[0] = n[0] * u2 + n[1] * v2 + n[2] * w2;
    vR[1] = t[0] * u2 + t[1] * v2 + t[2] * w2;
    vR[2] = m[0] * u2 + m[1] * v2 + m[2] * w2;
    bL[0] = n[0] * bx1 + n[1] * by1 + n[2] * bz1;
    bL[1] = t[0] * bx1 + t[1] * by1 + t[2] * bz1;
    bL[2] = m[0] * bx1 + m[1] * by1 + m[2] * bz1;
    bR[0] = n[0] * bx2 + n[1] * by2 + n[2] * bz2;
    bR[1] = t[0] * bx2 + t[1] * by2 + t[2] * bz2;
    bR[2] = m[0] * bx2 + m[1] * by2 + m[2] * bz2;

    // fast magnetosonic speeds of the two states
    const R aaL = bL[0] / sqrt(r1);
    const R b2L = bL[0] * bL[0] + bL[1] * bL[1] + bL[2] * bL[2];
    const R b21 = b2L / r1;
    const R cL = sqrt(gamma * p1 / r1);
    R qp = sqrt(b21 + cL * (cL + R(2) * aaL));
    R qm = sqrt(b21 + cL * (cL - R(2) * aaL));
    const R cfL = (qp + qm) / R(2);
    const R ptL = p1 + b2L / R(2);

    const R aaR = bR[0] / sqrt(r2);
    const R b2R = bR[0] * bR[0] + bR[1] * bR[1] + bR[2] * bR[2];
    const R b22 = b2R / r2;
    const R cR = sqrt(gamma * p2 / r2);
    qp = sqrt(b22 + cR * (cR + R(2) * aaR));
    qm = sqrt(b22 + cR * (cR - R(2) * aaR));
    const R cfR = (qp + qm) / R(2);
    const R ptR = p2 + b2R / R(2);

    const int n_disc = fl.left_ydar ? 2 : fl.n_disc;
    // speed of the averaged state: only the n_disc 1/2 estimates and Lax use it
    R cfC = R(0);
    if (n_state == 0 || n_disc == 1 || n_disc == 2) {
        const R ro = (r2 + r1) / R(2);
        const R ap = (p2 + p1) / R(2);
        const R aC = (aaL + aaR) / R(2);
        const R b2o = (b22 + b21) / R(2);
        const R cC = sqrt(gamma * ap / ro);
        const R qpc = sqrt(b2o + cC * (cC + R(2) * aC));
        const R qmc = sqrt(b2o + cC * (cC - R(2) * aC));
        cfC = (qpc + qmc) / R(2);
    }
    const R vC1 = (vL[0] + vR[0]) / R(2);

    R SL = R(0), SR = R(0);
    if (n_disc == 0) {
        SL = rmin(vL[0] - cfL, vR[0] - cfR);
        SR = rmax(vL[0] + cfL, vR[0] + cfR);
    } else if (n_disc == 1) {
        SL = rmin(vL[0] - cfL, vC1 - cfC);
        SR = rmax(vR[0] + cfR, vC1 + cfC);
    } else if (n_disc == 2) {
        const R SL_1 = rmin(vL[0] - cfL, vC1 - cfC);
        const R SR_1 = rmax(vR[0] + cfR, vC1 + cfC);
        const R SL_2 = rmin(vL[0] - cfL, vR[0] - cfR);
        const R SR_2 = rmax(vL[0] + cfL, vR[0] + cfR);
        const R oo = R(0.6);
        const R oo1 = R(1) - oo;
        SL = oo * SL_1 + oo1 * SL_2;
        SR = oo * SR_1 + oo1 * SR_2;
    } else if (n_disc == 3) {
        SL = rmin(vL[0], vR[0]) - rmax(cfL, cfR);
        SR = rmax(vL[0], vR[0]) + rmax(cfL, cfR);
    }
    dsr = SR;
    dsl = SL;

    const R suR = SR - vR[0];
    const R suL = SL - vL[0];
    const R SM = (suR * r2 * vR[0] - ptR + ptL - suL * r1 * vL[0]) / (suR * r2 - suL * r1);
    dsc = SM;
    if (fl.contact) wv = SM;

    if (n_state == 0) {
        const R TR0 = fabs(vL[0] + vR[0]) / R(2) + cfC;
        SR = TR0;
        SL = -TR0;
    }

    // energies and v.B of the two states (original Cartesian frame)
    const R sbv1 = u1 * bx1 + v1 * by1 + w1 * bz1;
    const R sbv2 = u2 * bx2 + v2 * by2 + w2 * bz2;
    auto energy1 = [&]() { return p1 / g1 + r1 * ((u1 * u1 + v1 * v1 + w1 * w1) / R(2)) + b2L / R(2); };
    auto energy2 = [&]() { return p2 / g1 + r2 * ((u2 * u2 + v2 * v2 + w2 * w2) / R(2)) + b2R / R(2); };

    R FLk[NK > 0 ? NK : 1], FRk[NK > 0 ? NK : 1];
#pragma unroll
    for (int i = 0; i < NK; ++i) {
        FLk[i] = kl[i] * vL[0];
        FRk[i] = kr[i] * vR[0];
    }

    R out[8];
    if (n_state <= 1) {  // Lax / HLL
        const R e1 = energy1(), e2 = energy2();
        R FL[8], FR[8], UL[8], UR[8], UZ[8];
        side_flux(r1, vL, bL, ptL, e1, sbv1, FL, UL);
        side_flux(r2, vR, bR, ptR, e2, sbv2, FR, UR);
#pragma unroll
        for (int k = 0; k < 8; ++k) UZ[k] = (SR * UR[k] - SL * UL[k] + FL[k] - FR[k]) / (SR - SL);
        if (fl.null_bn) UZ[5] = R(0);
        R UZk[NK > 0 ? NK : 1];
#pragma unroll
        for (int i = 0; i < NK; ++i) UZk[i] = (SR * kr[i] - SL * kl[i] + FLk[i] - FRk[i]) / (SR - SL);
        if (fl.left_ydar) wv = SL;
        R TL = SL, TR = SR;
        int wsel;  // state the face moves through: 0 left, 1 HLL average, 2 right
        if (SL > wv || fl.left_ydar) {
            TL = R(0);
            wsel = 0;
        } else if (SL <= wv && wv <= SR) {
            wsel = 1;
        } else if (SR < wv) {
            TR = R(0);
            wsel = 2;
        } else {
            return 1;
        }
        const R a = TR * TL;
        const R b = TR - TL;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const R Uw = wsel == 0 ? UL[k] : (wsel == 1 ? UZ[k] : UR[k]);
            out[k] = (TR * FL[k] - TL * FR[k] + a * (UR[k] - UL[k])) / b - wv * Uw;
        }
#pragma unroll
        for (int k = 0; k < NK; ++k) {
            const R Kw = wsel == 0 ? kl[k] : (wsel == 1 ? UZk[k] : kr[k]);
            kout[k] = (TR * FLk[k] - TL * FRk[k] + a * (kr[k] - kl[k])) / b - wv * Kw;
        }
    } else if (n_state == 2) {  // HLLC
        if (fl.left_ydar) wv = SL;
        int zone;
        if (SL >= wv || fl.left_ydar)
            zone = 1;
        else if (SL <= wv && SM >= wv)
            zone = 2;
        else if (SM <= wv && SR > wv)
            zone = 3;
        else if (SR <= wv)
            zone = 4;
        else
            return 2;
        const bool left = zone <= 2;
        const R e1 = energy1(), e2 = energy2();
        R FX[8], UX[8];
        if (left)
            side_flux(r1, vL, bL, ptL, e1, sbv1, FX, UX);
        else
            side_flux(r2, vR, bR, ptR, e2, sbv2, FX, UX);
        if (zone == 1 || zone == 4) {
            if (TRACK) {
                *upw = left ? 1 : 2;
                *wv_out = wv;
            }
#pragma unroll
            for (int k = 0; k < 8; ++k) out[k] = FX[k] - wv * UX[k];
#pragma unroll
            for (int k = 0; k < NK; ++k) kout[k] = (left ? FLk[k] : FRk[k]) - wv * (left ? kl[k] : kr[k]);
        } else {
            // HLL average state; component 4 is not used by HLLC
            R UL[8], UR[8], FL[8], FR[8], UZ[8];
            side_flux(r1, vL, bL, ptL, e1, sbv1, FL, UL);
            side_flux(r2, vR, bR, ptR, e2, sbv2, FR, UR);
#pragma unroll
            for (int k = 0; k < 8; ++k) UZ[k] = (SR * UR[k] - SL * UL[k] + FL[k] - FR[k]) / (SR - SL);
            if (fl.null_bn) UZ[5] = R(0);
            const R ptz = (suR * r2 * ptL - suL * r1 * ptR + r1 * r2 * suR * suL * (vR[0] - vL[0])) /
                          (suR * r2 - suL * r1);
            const R sbvz = (UZ[5] * UZ[1] + UZ[6] * UZ[2] + UZ[7] * UZ[3]) / UZ[0];
            const R S = left ? SL : SR;
            const R su = left ? suL : suR;
            const R rX = left ? r1 : r2;
            const R eX = left ? e1 : e2;
            const R ptX = left ? ptL : ptR;
            const R vX0 = left ? vL[0] : vR[0], vX1 = left ? vL[1] : vR[1], vX2 = left ? vL[2] : vR[2];
            const R bX1 = left ? bL[1] : bR[1], bX2 = left ? bL[2] : bR[2];
            const R sbvX = left ? sbv1 : sbv2;
            const R sum = su / (S - SM);
            const R rz = rX * sum;
            R vz1 = vX1 + UZ[5] * (bX1 - UZ[6]) / su / rX;
            R vz2 = vX2 + UZ[5] * (bX2 - UZ[7]) / su / rX;
            R bz1 = UZ[6], bz2 = UZ[7];
            const R ez = eX * sum + (ptz * SM - ptX * vX0 + UZ[5] * (sbvX - sbvz)) / (S - SM);
            if (fabs(UZ[5]) <= RConst<R>::epsb()) {
                vz1 = vX1;
                vz2 = vX2;
                bz1 = bX1 * sum;
                bz2 = bX2 * sum;
            }
            R UZX[8];
            UZX[0] = rz;
            UZX[1] = SM * rz;
            UZX[2] = vz1 * rz;
            UZX[3] = vz2 * rz;
            UZX[4] = ez;
            UZX[5] = UZ[5];
            UZX[6] = bz1;
            UZX[7] = bz2;
            out[0] = FX[0] + S * (rz - rX) - wv * UZX[0];
            out[4] = FX[4] + S * (ez - eX) - wv * UZX[4];
#pragma unroll
            for (int k = 1; k < 4; ++k) out[k] = FX[k] + S * (UZX[k] - UX[k]) - wv * UZX[k];
#pragma unroll
            for (int k = 5; k < 8; ++k) out[k] = FX[k] + S * (UZX[k] - UX[k]) - wv * UZX[k];
#pragma unroll
            for (int k = 0; k < NK; ++k) {
                const R K = left ? kl[k] : kr[k];
                kout[k] = (left ? FLk[k] : FRk[k]) + S * (K * sum - K) - wv * (K * sum);
            }
        }
    } else if (n_state == 3) {  // HLLD
        // normal field of the HLL average state (the flux of B_n is 0 on both sides)
        R bn = (SR * bR[0] - SL * bL[0] + R(0) - R(0)) / (SR - SL);
        if (fl.null_bn) bn = R(0);
        const R suRm = suR / (SR - SM);
        const R suLm = suL / (SL - SM);
        const R rzR = r2 * suRm;
        const R rzL = r1 * suLm;
        const R rzRs = sqrt(rzR);
        const R rzLs = sqrt(rzL);
        R SZL = SM - fabs(bn) / rzLs;
        R SZR = SM + fabs(bn) / rzRs;
        R sbn;
        bool ibn;
        if (fabs(bn) > RConst<R>::epsb()) {
            sbn = fabs(bn) / bn;
            ibn = true;
        } else {
            sbn = R(0);
            ibn = false;
            SZL = SM;
            SZR = SM;
        }
        if (fl.left_ydar) wv = SL;
        int zone = 0;  // replay of the reference's tests; later ones overwrite
        if (SL >= wv || fl.left_ydar)
            zone = 1;
        else if (SL <= wv && SZL >= wv)
            zone = 2;
        if (ibn) {
            if (SZL <= wv && SM >= wv)
                zone = 3;
            else if (SM <= wv && SZR >= wv)
                zone = 4;
        }
        if (SZR <= wv && SR >= wv)
            zone = 5;
        else if (SR <= wv)
            zone = 6;
        if (zone == 0) return 3;

        const bool left = zone <= 3;
        const R eX = left ? energy1() : energy2();
        R FX[8], UX[8];
        if (left)
            side_flux(r1, vL, bL, ptL, eX, sbv1, FX, UX);
        else
            side_flux(r2, vR, bR, ptR, eX, sbv2, FX, UX);
        if (zone == 1 || zone == 6) {
            if (TRACK) {
                *upw = left ? 1 : 2;
                *wv_out = wv;
            }
#pragma unroll
            for (int k = 0; k < 8; ++k) out[k] = FX[k] - wv * UX[k];
#pragma unroll
            for (int k = 0; k < NK; ++k) kout[k] = (left ? FLk[k] : FRk[k]) - wv * (left ? kl[k] : kr[k]);
        } else {
            const R ptz = (suR * r2 * ptL - suL * r1 * ptR + r1 * r2 * suR * suL * (vR[0] - vL[0])) /
                          (suR * r2 - suL * r1);
            const R bn2 = bn * bn;
            // single-star velocity / field of the left (zones 2, 3, 4) and right (3, 4, 5) states
            R vzL1 = R(0), vzL2 = R(0), bzL1 = R(0), bzL2 = R(0);
            R vzR1 = R(0), vzR2 = R(0), bzR1 = R(0), bzR2 = R(0);
            if (zone != 5) {
                R tvL, tbL;
                const R ttL = r1 * suL * (SL - SM) - bn2;
                if (fabs(ttL) < RConst<R>::tt_eps()) {
                    tvL = R(0);
                    tbL = R(0);
                } else {
                    tvL = (SM - vL[0]) / ttL;
                    tbL = (r1 * suL * suL - bn2) / ttL;
                }
                vzL1 = vL[1] - bn * bL[1] * tvL;
                vzL2 = vL[2] - bn * bL[2] * tvL;
                bzL1 = bL[1] * tbL;
                bzL2 = bL[2] * tbL;
            }
            if (zone != 2) {
                R tvR, tbR;
                const R ttR = r2 * suR * (SR - SM) - bn2;
                if (fabs(ttR) < RConst<R>::tt_eps()) {
                    tvR = R(0);
                    tbR = R(0);
                } else {
                    tvR = (SM - vR[0]) / ttR;
                    tbR = (r2 * suR * suR - bn2) / ttR;
                }
                vzR1 = vR[1] - bn * bR[1] * tvR;
                vzR2 = vR[2] - bn * bR[2] * tvR;
                bzR1 = bR[1] * tbR;
                bzR2 = bR[2] * tbR;
            }
            // single-star state of the side the zone belongs to
            const R vz1 = left ? vzL1 : vzR1, vz2 = left ? vzL2 : vzR2;
            const R bz1 = left ? bzL1 : bzR1, bz2 = left ? bzL2 : bzR2;
            const R sbvX = bn * SM + bz1 * vz1 + bz2 * vz2;
            const R rz = left ? rzL : rzR;
            const R sum = left ? suLm : suRm;
            const R S = left ? SL : SR;
            const R ez = eX * sum + (ptz * SM - (left ? ptL : ptR) * (left ? vL[0] : vR[0]) +
                                     bn * ((left ? sbv1 : sbv2) - sbvX)) /
                                        (S - SM);
            R UZX[8];
            UZX[0] = rz;
            UZX[1] = SM * rz;
            UZX[2] = vz1 * rz;
            UZX[3] = vz2 * rz;
            UZX[4] = ez;
            UZX[5] = bn;
            UZX[6] = bz1;
            UZX[7] = bz2;
            if (zone == 2 || zone == 5) {
#pragma unroll
                for (int k = 0; k < 8; ++k) out[k] = FX[k] + S * (UZX[k] - UX[k]) - wv * UZX[k];
#pragma unroll
                for (int k = 0; k < NK; ++k) {
                    const R K = left ? kl[k] : kr[k];
                    kout[k] = (left ? FLk[k] : FRk[k]) + S * (K * sum - K) - wv * (K * sum);
                }
            } else {
                // double-star state (rho** = rho*, v**_n = SM)
                const R rzss = rzRs + rzLs;
                const R rzps = rzRs * rzLs;
                const R vzz1 = (rzLs * vzL1 + rzRs * vzR1 + sbn * (bzR1 - bzL1)) / rzss;
                const R vzz2 = (rzLs * vzL2 + rzRs * vzR2 + sbn * (bzR2 - bzL2)) / rzss;
                const R bzz1 = (rzLs * bzR1 + rzRs * bzL1 + sbn * rzps * (vzR1 - vzL1)) / rzss;
                const R bzz2 = (rzLs * bzR2 + rzRs * bzL2 + sbn * rzps * (vzR2 - vzL2)) / rzss;
                const R sbzz = bn * SM + bzz1 * vzz1 + bzz2 * vzz2;
                const R ezz = left ? ez - rzLs * sbn * (sbvX - sbzz) : ez + rzRs * sbn * (sbvX - sbzz);
                const R SZ = left ? SZL : SZR;
                R UZZ[8];
                UZZ[0] = rz;
                UZZ[1] = SM * rz;
                UZZ[2] = vzz1 * rz;
                UZZ[3] = vzz2 * rz;
                UZZ[4] = ezz;
                UZZ[5] = bn;
                UZZ[6] = bzz1;
                UZZ[7] = bzz2;
#pragma unroll
                for (int k = 0; k < 8; ++k)
                    out[k] = FX[k] + SZ * (UZZ[k] - UZX[k]) + S * (UZX[k] - UX[k]) - wv * UZZ[k];
#pragma unroll
                for (int k = 0; k < NK; ++k) {
                    const R K = left ? kl[k] : kr[k];
                    const R qz = K * sum;
                    kout[k] = (left ? FLk[k] : FRk[k]) + SZ * (qz - qz) + S * (qz - K) - wv * qz;
                }
            }
        }
    } else {
        return 4;
    }
    R SN, wbn;
    SN = rmax(fabs(SL), fabs(SR));
    if (n_state <= 1) {
        if (wv >= SR)
            wbn = wv * bR[0];
        else if (wv <= SL)
            wbn = wv * bL[0];
        else
            wbn = wv * (bL[0] + bR[0]) / R(2);
    } else {
        if (wv > SR)
            wbn = wv * bR[0];
        else if (wv < SL)
            wbn = wv * bL[0];
        else
            wbn = wv * (bL[0] + bR[0]) / R(2);
    }
    const R qb0 = fl.null_bn ? R(0) : -SN * (bR[0] - bL[0]) - wbn;
    qout[0] = out[0];
    qout[4] = out[4];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        qout[i + 1] = n[i] * out[1] + t[i] * out[2] + m[i] * out[3];
        qout[i + 5] = spi4 * (n[i] * qb0 + t[i] * out[6] + m[i] * out[7]);
    }
    return 0;
}

// Flux through a face that lies wholly in one side's wave region (HLLC zones
// 1/4, HLLD zones 1/6): the physical flux of that side minus wv U, with the
// normal-B term -SN (bR - bL) - wv bn of riemann_flux, evaluated in FP64 from
// the FP64 face states. The FP32 solver supplies the region (left), the frame
// speed wv and the wave speeds SL, SR. Supersonic faces, where the upwind
// state's flux is the whole answer, thus keep FP64 accuracy in the
// mixed-precision step. The flux is formed directly in Cartesian components
// (the face basis cancels out of an upwind flux), so this path is an ulp or
// so from the FP64 solver's rotated result, not bit-matched to it.
template <int NK>
__device__ __forceinline__ void upwind_flux_fp64(const double nrm[3], double wv, const double* q1, const double* q2,
                                                 const double* kl, const double* kr, bool left, double SL, double SR,
                                                 bool null_bn, double gamma, double* qout, double* kout) {
    const double spi4 = RConst<double>::spi4();
    const double ispi4 = 1.0 / 3.5449077018110318;
    const double ig1 = 1.0 / (gamma - 1.0);
    const double* q = left ? q1 : q2;
    const double r = q[0], v0 = q[1], v1 = q[2], v2 = q[3], p = q[4];
    const double B0 = q[5] * ispi4, B1 = q[6] * ispi4, B2 = q[7] * ispi4;
    const double vn = nrm[0] * v0 + nrm[1] * v1 + nrm[2] * v2;
    const double bn = nrm[0] * B0 + nrm[1] * B1 + nrm[2] * B2;
    const double b2 = B0 * B0 + B1 * B1 + B2 * B2;
    const double pt = p + b2 * 0.5;
    const double vb = v0 * B0 + v1 * B1 + v2 * B2;
    const double e = p * ig1 + r * ((v0 * v0 + v1 * v1 + v2 * v2) * 0.5) + b2 * 0.5;
    const double rvw = r * (vn - wv);
    qout[0] = rvw;
    qout[1] = rvw * v0 + pt * nrm[0] - bn * B0;
    qout[2] = rvw * v1 + pt * nrm[1] - bn * B1;
    qout[3] = rvw * v2 + pt * nrm[2] - bn * B2;
    qout[4] = (e + pt) * vn - bn * vb - wv * e;
#pragma unroll
    for (int k = 0; k < NK; ++k) {
        const double K = left ? kl[k] : kr[k];
        kout[k] = K * vn - wv * K;
    }
    const double bL0 = (nrm[0] * q1[5] + nrm[1] * q1[6] + nrm[2] * q1[7]) * ispi4;
    const double bR0 = (nrm[0] * q2[5] + nrm[1] * q2[6] + nrm[2] * q2[7]) * ispi4;
    const double SN = rmax(fabs(SL), fabs(SR));
    double wbn;
    if (wv > SR)
        wbn = wv * bR0;
    else if (wv < SL)
        wbn = wv * bL0;
    else
        wbn = wv * (bL0 + bR0) * 0.5;
    const double qb0 = null_bn ? 0.0 : -SN * (bR0 - bL0) - wbn;
    // tangential part of (vn B - bn v - wv B) plus qb0 along the normal
    const double tb = -wv * bn;  // normal component of (vn B - bn v - wv B)
    const double Bv[3] = {B0, B1, B2}, vv[3] = {v0, v1, v2};
#pragma unroll
    for (int i = 0; i < 3; ++i) qout[5 + i] = spi4 * (nrm[i] * qb0 + (vn * Bv[i] - bn * vv[i] - wv * Bv[i] - tb * nrm[i]));
}

}  // namespace titan
