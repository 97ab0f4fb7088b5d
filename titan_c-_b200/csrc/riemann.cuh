// Device-side MHD Riemann solvers for one moving face.
//
// Computes what TITAN's Phys_param::chlld (TITAN/source/Phys_param.cpp:882-1878)
// computes: the Lax (n_state 0), HLL (1), HLLC (2) and HLLD (3) fluxes in the
// frame of a face moving with normal speed w, rotated into the face basis of
// get_bazis (TITAN/source/Help_funk.cpp:219-232), with the Powell-form normal
// B flux -SN*(bR-bL) - w*bn and the sqrt(4*pi) Gaussian rescale of B.
//
// The arithmetic is written so that, in double precision and compiled without
// FMA contraction (the FP64 translation unit uses -fmad=false), every value
// rounds exactly as the reference's x86-64 build does: same expression trees,
// same branch order (including the HLLD zone-5 overwrite when |bn| <= epsb and
// the Lax speeds that replace SL/SR after dsl/dsr were recorded). The single
// precision instantiation runs the same algorithm in float.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace titan {

template <typename R>
struct RConst;
template <>
struct RConst<double> {
    // sqrt(4*pi) rounded to double, as TITAN/source/Header.h:99 computes it
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

// Returns 0 on success; 1/2/3 where the reference would abort (no admissible
// wave region, i.e. NaN speeds) for the HLL/HLLC/HLLD branches, 4 for a bad
// n_state. q1/q2: rho, u, v, w, p, Bx, By, Bz (Gaussian B). qout: 8 fluxes.
// kl/kr/kout: NK passive scalars carried by the contact.
template <typename R, int NK>
__device__ __forceinline__ int riemann_flux(int n_state, const R nrm[3], R w, const R* q1, const R* q2,
                                            const R* kl, const R* kr, R* qout, R* kout, R& dsl, R& dsc,
                                            R& dsr, RiemannFlags fl, R gamma) {
    const R spi4 = RConst<R>::spi4();
    const R g1 = gamma - R(1);
    R wv = w;
    const R r1 = q1[0], u1 = q1[1], v1 = q1[2], w1 = q1[3], p1 = q1[4];
    const R bx1 = q1[5] / spi4, by1 = q1[6] / spi4, bz1 = q1[7] / spi4;
    const R r2 = q2[0], u2 = q2[1], v2 = q2[2], w2 = q2[3], p2 = q2[4];
    const R bx2 = q2[5] / spi4, by2 = q2[6] / spi4, bz2 = q2[7] / spi4;
    const R ro = (r2 + r1) / R(2);
    const R ap = (p2 + p1) / R(2);

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

    // fast magnetosonic speeds of the two states and of their average
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

    const R aC = (aaL + aaR) / R(2);
    const R b2o = (b22 + b21) / R(2);
    const R cC = sqrt(gamma * ap / ro);
    qp = sqrt(b2o + cC * (cC + R(2) * aC));
    qm = sqrt(b2o + cC * (cC - R(2) * aC));
    const R cfC = (qp + qm) / R(2);
    const R vC1 = (vL[0] + vR[0]) / R(2);

    R SL = R(0), SR = R(0);
    const int n_disc = fl.left_ydar ? 2 : fl.n_disc;
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

    const R upt1 = (u1 * u1 + v1 * v1 + w1 * w1) / R(2);
    const R sbv1 = u1 * bx1 + v1 * by1 + w1 * bz1;
    const R upt2 = (u2 * u2 + v2 * v2 + w2 * w2) / R(2);
    const R sbv2 = u2 * bx2 + v2 * by2 + w2 * bz2;
    const R e1 = p1 / g1 + r1 * upt1 + b2L / R(2);
    const R e2 = p2 / g1 + r2 * upt2 + b2R / R(2);

    R FL[8], FR[8], UL[8], UR[8], UZ[8];
    FL[0] = r1 * vL[0];
    FL[1] = r1 * vL[0] * vL[0] + ptL - bL[0] * bL[0];
    FL[2] = r1 * vL[0] * vL[1] - bL[0] * bL[1];
    FL[3] = r1 * vL[0] * vL[2] - bL[0] * bL[2];
    FL[4] = (e1 + ptL) * vL[0] - bL[0] * sbv1;
    FL[5] = R(0);
    FL[6] = vL[0] * bL[1] - vL[1] * bL[0];
    FL[7] = vL[0] * bL[2] - vL[2] * bL[0];
    FR[0] = r2 * vR[0];
    FR[1] = r2 * vR[0] * vR[0] + ptR - bR[0] * bR[0];
    FR[2] = r2 * vR[0] * vR[1] - bR[0] * bR[1];
    FR[3] = r2 * vR[0] * vR[2] - bR[0] * bR[2];
    FR[4] = (e2 + ptR) * vR[0] - bR[0] * sbv2;
    FR[5] = R(0);
    FR[6] = vR[0] * bR[1] - vR[1] * bR[0];
    FR[7] = vR[0] * bR[2] - vR[2] * bR[0];
    UL[0] = r1;
    UL[4] = e1;
    UR[0] = r2;
    UR[4] = e2;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        UL[i + 1] = r1 * vL[i];
        UL[i + 5] = bL[i];
        UR[i + 1] = r2 * vR[i];
        UR[i + 5] = bR[i];
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) UZ[k] = (SR * UR[k] - SL * UL[k] + FL[k] - FR[k]) / (SR - SL);

    R FLk[NK > 0 ? NK : 1], FRk[NK > 0 ? NK : 1], UZk[NK > 0 ? NK : 1];
#pragma unroll
    for (int i = 0; i < NK; ++i) {
        FLk[i] = kl[i] * vL[0];
        FRk[i] = kr[i] * vR[0];
        UZk[i] = (SR * kr[i] - SL * kl[i] + FLk[i] - FRk[i]) / (SR - SL);
    }
    if (fl.null_bn) UZ[5] = R(0);

    R qv[3], qb[3];
    R SN, wbn;

    if (n_state <= 1) {
        R FW[8], FWk[NK > 0 ? NK : 1];
        if (fl.left_ydar) wv = SL;
        R TL = SL, TR = SR;
        if (SL > wv || fl.left_ydar) {
            TL = R(0);
#pragma unroll
            for (int k = 0; k < 8; ++k) FW[k] = wv * UL[k];
#pragma unroll
            for (int k = 0; k < NK; ++k) FWk[k] = wv * kl[k];
        } else if (SL <= wv && wv <= SR) {
#pragma unroll
            for (int k = 0; k < 8; ++k) FW[k] = wv * UZ[k];
#pragma unroll
            for (int k = 0; k < NK; ++k) FWk[k] = wv * UZk[k];
        } else if (SR < wv) {
            TR = R(0);
#pragma unroll
            for (int k = 0; k < 8; ++k) FW[k] = wv * UR[k];
#pragma unroll
            for (int k = 0; k < NK; ++k) FWk[k] = wv * kr[k];
        } else {
            return 1;
        }
        const R a = TR * TL;
        const R b = TR - TL;
        qout[0] = (TR * FL[0] - TL * FR[0] + a * (UR[0] - UL[0])) / b - FW[0];
        qout[4] = (TR * FL[4] - TL * FR[4] + a * (UR[4] - UL[4])) / b - FW[4];
#pragma unroll
        for (int k = 0; k < NK; ++k) kout[k] = (TR * FLk[k] - TL * FRk[k] + a * (kr[k] - kl[k])) / b - FWk[k];
#pragma unroll
        for (int k = 1; k < 4; ++k) qv[k - 1] = (TR * FL[k] - TL * FR[k] + a * (UR[k] - UL[k])) / b - FW[k];
#pragma unroll
        for (int k = 5; k < 8; ++k) qb[k - 5] = (TR * FL[k] - TL * FR[k] + a * (UR[k] - UL[k])) / b - FW[k];
        SN = rmax(fabs(SL), fabs(SR));
        if (wv >= SR)
            wbn = wv * bR[0];
        else if (wv <= SL)
            wbn = wv * bL[0];
        else
            wbn = wv * (bL[0] + bR[0]) / R(2);
    } else if (n_state == 2) {
        const R suRm = suR / (SR - SM);
        const R suLm = suL / (SL - SM);
        const R rzR = r2 * suRm;
        const R rzL = r1 * suLm;
        const R ptz = (suR * r2 * ptL - suL * r1 * ptR + r1 * r2 * suR * suL * (vR[0] - vL[0])) /
                      (suR * r2 - suL * r1);
        R vzR1 = vR[1] + UZ[5] * (bR[1] - UZ[6]) / suR / r2;
        R vzR2 = vR[2] + UZ[5] * (bR[2] - UZ[7]) / suR / r2;
        R vzL1 = vL[1] + UZ[5] * (bL[1] - UZ[6]) / suL / r1;
        R vzL2 = vL[2] + UZ[5] * (bL[2] - UZ[7]) / suL / r1;
        R bzR1 = UZ[6], bzR2 = UZ[7], bzL1 = UZ[6], bzL2 = UZ[7];
        const R sbvz = (UZ[5] * UZ[1] + UZ[6] * UZ[2] + UZ[7] * UZ[3]) / UZ[0];
        const R ezR = e2 * suRm + (ptz * SM - ptR * vR[0] + UZ[5] * (sbv2 - sbvz)) / (SR - SM);
        const R ezL = e1 * suLm + (ptz * SM - ptL * vL[0] + UZ[5] * (sbv1 - sbvz)) / (SL - SM);
        if (fabs(UZ[5]) <= RConst<R>::epsb()) {
            vzR1 = vR[1];
            vzR2 = vR[2];
            vzL1 = vL[1];
            vzL2 = vL[2];
            bzR1 = bR[1] * suRm;
            bzR2 = bR[2] * suRm;
            bzL1 = bL[1] * suLm;
            bzL2 = bL[2] * suLm;
        }
        R UZL[8], UZR[8];
        UZL[0] = rzL;
        UZL[4] = ezL;
        UZR[0] = rzR;
        UZR[4] = ezR;
        UZL[1] = SM * rzL;
        UZL[2] = vzL1 * rzL;
        UZL[3] = vzL2 * rzL;
        UZR[1] = SM * rzR;
        UZR[2] = vzR1 * rzR;
        UZR[3] = vzR2 * rzR;
        UZL[5] = UZ[5];
        UZL[6] = bzL1;
        UZL[7] = bzL2;
        UZR[5] = UZ[5];
        UZR[6] = bzR1;
        UZR[7] = bzR2;
        if (fl.left_ydar) wv = SL;
        R out[8];
        if (SL >= wv || fl.left_ydar) {
#pragma unroll
            for (int k = 0; k < 8; ++k) out[k] = FL[k] - wv * UL[k];
#pragma unroll
            for (int k = 0; k < NK; ++k) kout[k] = FLk[k] - wv * kl[k];
        } else if (SL <= wv && SM >= wv) {
            out[0] = FL[0] + SL * (rzL - r1) - wv * UZL[0];
            out[4] = FL[4] + SL * (ezL - e1) - wv * UZL[4];
#pragma unroll
            for (int k = 0; k < NK; ++k) kout[k] = FLk[k] + SL * (kl[k] * suLm - kl[k]) - wv * (kl[k] * suLm);
#pragma unroll
            for (int k = 1; k < 4; ++k) out[k] = FL[k] + SL * (UZL[k] - UL[k]) - wv * UZL[k];
#pragma unroll
            for (int k = 5; k < 8; ++k) out[k] = FL[k] + SL * (UZL[k] - UL[k]) - wv * UZL[k];
        } else if (SM <= wv && SR > wv) {
            out[0] = FR[0] + SR * (rzR - r2) - wv * UZR[0];
            out[4] = FR[4] + SR * (ezR - e2) - wv * UZR[4];
#pragma unroll
            for (int k = 0; k < NK; ++k) kout[k] = FRk[k] + SR * (kr[k] * suRm - kr[k]) - wv * (kr[k] * suRm);
#pragma unroll
            for (int k = 1; k < 4; ++k) out[k] = FR[k] + SR * (UZR[k] - UR[k]) - wv * UZR[k];
#pragma unroll
            for (int k = 5; k < 8; ++k) out[k] = FR[k] + SR * (UZR[k] - UR[k]) - wv * UZR[k];
        } else if (SR <= wv) {
#pragma unroll
            for (int k = 0; k < 8; ++k) out[k] = FR[k] - wv * UR[k];
#pragma unroll
            for (int k = 0; k < NK; ++k) kout[k] = FRk[k] - wv * kr[k];
        } else {
            return 2;
        }
        qout[0] = out[0];
        qout[4] = out[4];
        qv[0] = out[1];
        qv[1] = out[2];
        qv[2] = out[3];
        qb[0] = out[5];
        qb[1] = out[6];
        qb[2] = out[7];
        SN = rmax(fabs(SL), fabs(SR));
        if (wv > SR)
            wbn = wv * bR[0];
        else if (wv < SL)
            wbn = wv * bL[0];
        else
            wbn = wv * (bL[0] + bR[0]) / R(2);
    } else if (n_state == 3) {
        const R ptz = (suR * r2 * ptL - suL * r1 * ptR + r1 * r2 * suR * suL * (vR[0] - vL[0])) /
                      (suR * r2 - suL * r1);
        const R suRm = suR / (SR - SM);
        const R suLm = suL / (SL - SM);
        const R rzR = r2 * suRm;
        const R rzL = r1 * suLm;
        const R bn = UZ[5];
        const R bn2 = bn * bn;
        R tvR, tbR, tvL, tbL;
        const R ttR = r2 * suR * (SR - SM) - bn2;
        if (fabs(ttR) < RConst<R>::tt_eps()) {
            tvR = R(0);
            tbR = R(0);
        } else {
            tvR = (SM - vR[0]) / ttR;
            tbR = (r2 * suR * suR - bn2) / ttR;
        }
        const R ttL = r1 * suL * (SL - SM) - bn2;
        if (fabs(ttL) < RConst<R>::tt_eps()) {
            tvL = R(0);
            tbL = R(0);
        } else {
            tvL = (SM - vL[0]) / ttL;
            tbL = (r1 * suL * suL - bn2) / ttL;
        }
        const R vzL1 = vL[1] - bn * bL[1] * tvL;
        const R vzL2 = vL[2] - bn * bL[2] * tvL;
        const R vzR1 = vR[1] - bn * bR[1] * tvR;
        const R vzR2 = vR[2] - bn * bR[2] * tvR;
        const R bzL1 = bL[1] * tbL;
        const R bzL2 = bL[2] * tbL;
        const R bzR1 = bR[1] * tbR;
        const R bzR2 = bR[2] * tbR;
        const R sbvL = bn * SM + bzL1 * vzL1 + bzL2 * vzL2;
        const R sbvR = bn * SM + bzR1 * vzR1 + bzR2 * vzR2;
        const R ezR = e2 * suRm + (ptz * SM - ptR * vR[0] + bn * (sbv2 - sbvR)) / (SR - SM);
        const R ezL = e1 * suLm + (ptz * SM - ptL * vL[0] + bn * (sbv1 - sbvL)) / (SL - SM);
        const R rzRs = sqrt(rzR);
        const R rzLs = sqrt(rzL);
        const R rzss = rzRs + rzLs;
        const R rzps = rzRs * rzLs;
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
        const R vzz1 = (rzLs * vzL1 + rzRs * vzR1 + sbn * (bzR1 - bzL1)) / rzss;
        const R vzz2 = (rzLs * vzL2 + rzRs * vzR2 + sbn * (bzR2 - bzL2)) / rzss;
        const R bzz1 = (rzLs * bzR1 + rzRs * bzL1 + sbn * rzps * (vzR1 - vzL1)) / rzss;
        const R bzz2 = (rzLs * bzR2 + rzRs * bzL2 + sbn * rzps * (vzR2 - vzL2)) / rzss;
        const R sbzz = bn * SM + bzz1 * vzz1 + bzz2 * vzz2;
        const R ezzR = ezR + rzRs * sbn * (sbvR - sbzz);
        const R ezzL = ezL - rzLs * sbn * (sbvL - sbzz);

        // Star (UZ*) and double-star (UZZ*) states; the reference keeps
        // rho** = rho* and v**_n = SM.
        R UZL[8], UZR[8], UZZL[8], UZZR[8];
        UZL[0] = rzL;
        UZL[1] = SM * rzL;
        UZL[2] = vzL1 * rzL;
        UZL[3] = vzL2 * rzL;
        UZL[4] = ezL;
        UZL[5] = bn;
        UZL[6] = bzL1;
        UZL[7] = bzL2;
        UZR[0] = rzR;
        UZR[1] = SM * rzR;
        UZR[2] = vzR1 * rzR;
        UZR[3] = vzR2 * rzR;
        UZR[4] = ezR;
        UZR[5] = bn;
        UZR[6] = bzR1;
        UZR[7] = bzR2;
        UZZL[0] = rzL;
        UZZL[1] = SM * rzL;
        UZZL[2] = vzz1 * rzL;
        UZZL[3] = vzz2 * rzL;
        UZZL[4] = ezzL;
        UZZL[5] = bn;
        UZZL[6] = bzz1;
        UZZL[7] = bzz2;
        UZZR[0] = rzR;
        UZZR[1] = SM * rzR;
        UZZR[2] = vzz1 * rzR;
        UZZR[3] = vzz2 * rzR;
        UZZR[4] = ezzR;
        UZZR[5] = bn;
        UZZR[6] = bzz1;
        UZZR[7] = bzz2;

        if (fl.left_ydar) wv = SL;
        int zone = 0;  // the reference's j_ccs: 1..6, later tests overwrite earlier ones
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

        R out[8];
        const R* FX = (zone <= 3) ? FL : FR;
        const R* UX = (zone <= 3) ? UL : UR;
        const R* KX = (zone <= 3) ? kl : kr;
        if (zone == 1 || zone == 6) {
#pragma unroll
            for (int k = 0; k < 8; ++k) out[k] = FX[k] - wv * UX[k];
#pragma unroll
            for (int k = 0; k < NK; ++k) kout[k] = (zone == 1 ? FLk[k] : FRk[k]) - wv * KX[k];
        } else if (zone == 2 || zone == 5) {
            const R* UZX = (zone == 2) ? UZL : UZR;
            const R S = (zone == 2) ? SL : SR;
            const R sm = (zone == 2) ? suLm : suRm;
#pragma unroll
            for (int k = 0; k < 8; ++k) out[k] = FX[k] + S * (UZX[k] - UX[k]) - wv * UZX[k];
#pragma unroll
            for (int k = 0; k < NK; ++k)
                kout[k] = (zone == 2 ? FLk[k] : FRk[k]) + S * (KX[k] * sm - KX[k]) - wv * (KX[k] * sm);
        } else {
            const R* UZX = (zone == 3) ? UZL : UZR;
            const R* UZZX = (zone == 3) ? UZZL : UZZR;
            const R S = (zone == 3) ? SL : SR;
            const R SZ = (zone == 3) ? SZL : SZR;
            const R sm = (zone == 3) ? suLm : suRm;
#pragma unroll
            for (int k = 0; k < 8; ++k) out[k] = FX[k] + SZ * (UZZX[k] - UZX[k]) + S * (UZX[k] - UX[k]) - wv * UZZX[k];
#pragma unroll
            for (int k = 0; k < NK; ++k) {
                const R qz = KX[k] * sm;
                kout[k] = (zone == 3 ? FLk[k] : FRk[k]) + SZ * (qz - qz) + S * (qz - KX[k]) - wv * qz;
            }
        }
        qout[0] = out[0];
        qout[4] = out[4];
        qv[0] = out[1];
        qv[1] = out[2];
        qv[2] = out[3];
        qb[0] = out[5];
        qb[1] = out[6];
        qb[2] = out[7];
        SN = rmax(fabs(SL), fabs(SR));
        if (wv > SR)
            wbn = wv * bR[0];
        else if (wv < SL)
            wbn = wv * bL[0];
        else
            wbn = wv * (bL[0] + bR[0]) / R(2);
    } else {
        return 4;
    }
    qb[0] = -SN * (bR[0] - bL[0]) - wbn;
    if (fl.null_bn) qb[0] = R(0);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        qout[i + 1] = n[i] * qv[0] + t[i] * qv[1] + m[i] * qv[2];
        qout[i + 5] = spi4 * (n[i] * qb[0] + t[i] * qb[1] + m[i] * qb[2]);
    }
    return 0;
}

}  // namespace titan
