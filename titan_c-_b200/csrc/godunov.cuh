// Exact gas-dynamic Godunov solver of the heliopause (HP) faces when the
// magnetic pressure is folded into p there (bn_in_p_on_HP): the reference's
// Phys_param::Godunov_Solver_Alexashov (TITAN/source/Phys_param.cpp:1938-2385)
// with its Newton (:2387-2442), bisection (:2444-2519) and pressure-function
// (:2521-2536) helpers, in FP64 with the reference's expression trees (the
// face kernels built with -fmad=false reproduce it; the FP32 face kernels use
// it in FP64 too, since its iterations stop at a 1e-12 relative change). The
// reference's parenthesised macros (ga, g1 = ga - 1, g2 = ga + 1,
// gp = (g2 / ga) / 2, gm = (g1 / ga) / 2) are formed once. Where the reference
// exits this returns 1 (negative pressure in Newton), 2 (Newton without
// convergence after 1100 iterations), 3 (bisection likewise) or 4 (no wave
// pattern applies: non-finite input). q1, q2: rho, u, v, w, p; out: 5 fluxes
// (mass, momentum, energy) in the frame of a face moving at w; ds: dsl, dsc,
// dsr.
#pragma once

#include "riemann.cuh"
#include "step_types.h"

namespace titan {

constexpr double kGodunovEps = 1E-12;  // Header.h: eps

struct GodunovK {
    double ga, g1, g2, gp, gm;
    __device__ explicit GodunovK(double gamma)
        : ga(gamma), g1(gamma - 1.0), g2(gamma + 1.0), gp(((gamma + 1.0) / gamma) / 2.0),
          gm(((gamma - 1.0) / gamma) / 2.0) {}
};

__device__ __forceinline__ double gd_lev(const GodunovK& K, double enI, double pI, double rI, double enII, double pII, double rII, double uuu) {
    const double cI = sqrt(K.ga * pI / rI);
    const double cII = sqrt(K.ga * pII / rII);
    const double fI = (uuu - pI) / (rI * cI * sqrt(K.gp * uuu / pI + K.gm));
    const double fII = 2.0 / K.g1 * cII * (pow((uuu / pII), K.gm) - 1.0);
    const double f1 = fI + fII;
    const double f2 = enI - enII;
    return f1 - f2;
}

__device__ __forceinline__ int gd_newton(const GodunovK& K, double enI, double pI, double rI, double enII, double pII, double rII, double& p) {
    const double cI = sqrt(K.ga * pI / rI);
    const double cII = sqrt(K.ga * pII / rII);
    double pn = pI * rII * cII + pII * rI * cI + (enI - enII) * rI * cI * rII * cII;
    pn = pn / (rI * cI + rII * cII);
    const double pee = pn;
    int kiter = 0;
    while (true) {
        p = pn;
        if (p <= 0.0) return 1;
        kiter = kiter + 1;
        const double fI = (p - pI) / (rI * cI * sqrt(K.gp * p / pI + K.gm));
        double fIs = (K.ga + 1.0) * p / pI + (3.0 * K.ga - 1.0);
        fIs = fIs / (4.0 * K.ga * rI * cI * pow((K.gp * p / pI + K.gm), (3.0 / 2.0)));
        const double fII = (p - pII) / (rII * cII * sqrt(K.gp * p / pII + K.gm));
        double fIIs = (K.ga + 1.0) * p / pII + (3.0 * K.ga - 1.0);
        fIIs = fIIs / (4.0 * K.ga * rII * cII * pow((K.gp * p / pII + K.gm), (3.0 / 2.0)));
        if (kiter == 1100) return 2;
        pn = p - (fI + fII - (enI - enII)) / (fIs + fIIs);
        if (!(fabs(pn / pee - p / pee) >= kGodunovEps)) break;
    }
    p = pn;
    return 0;
}

__device__ __forceinline__ int gd_devtwo(const GodunovK& K, double enI, double pI, double rI, double enII, double pII, double rII, double& p) {
    const double epsil = 10e-10;
    double kl = pI, kp = pII;
    double ksi = gd_lev(K, enI, pI, rI, enII, pII, rII, kl);
    double ksir = gd_lev(K, enI, pI, rI, enII, pII, rII, kp);
    if (fabs(ksi) <= epsil) {
        p = kl;
        return 0;
    }
    if (fabs(ksir) <= epsil) {
        p = kp;
        return 0;
    }
    int kpizd = 0;
    while (true) {
        kpizd = kpizd + 1;
        if (kpizd == 1100) return 3;
        const double kc = (kl + kp) / 2.0;
        const double ksit = gd_lev(K, enI, pI, rI, enII, pII, rII, kc);
        if (fabs(ksit) <= epsil) {
            p = kc;
            return 0;
        }
        if ((ksi * ksit) <= 0.0) {
            kp = kc;
            ksir = ksit;
        } else {
            kl = kc;
            ksi = ksit;
        }
    }
}

__device__ __forceinline__ int godunov_exact(const double* nrm, double w, const double* q1, const double* q2, int contact, double gamma,
              double* out, double* ds) {
    const GodunovK K(gamma);
    const double al = nrm[0], be = nrm[1], ge = nrm[2];
    double t[3], m[3];
    {
        double nn[3] = {nrm[0], nrm[1], nrm[2]};
        face_basis(nn, t, m);
    }
    const double al2 = t[0], be2 = t[1], ge2 = t[2], al3 = m[0], be3 = m[1], ge3 = m[2];
    double enI = al * q1[1] + be * q1[2] + ge * q1[3];
    double teI2 = al2 * q1[1] + be2 * q1[2] + ge2 * q1[3];
    double teI3 = al3 * q1[1] + be3 * q1[2] + ge3 * q1[3];
    double enII = al * q2[1] + be * q2[2] + ge * q2[3];
    double teII2 = al2 * q2[1] + be2 * q2[2] + ge2 * q2[3];
    double teII3 = al3 * q2[1] + be3 * q2[2] + ge3 * q2[3];
    double pI = q1[4], pII = q2[4], rI = q1[0], rII = q2[0];
    int ipiz = 0;
    if (pI > pII) {  // the higher pressure on the right
        const double eno2 = enII, teo22 = teII2, teo23 = teII3, p2 = pII, r2 = rII;
        const double eno1 = enI, teo12 = teI2, teo13 = teI3, p1 = pI, r1 = rI;
        enI = -eno2;
        teI2 = teo22;
        teI3 = teo23;
        pI = p2;
        rI = r2;
        enII = -eno1;
        teII2 = teo12;
        teII3 = teo13;
        pII = p1;
        rII = r1;
        w = -w;
        ipiz = 1;
    }
    double cI = 0.0, cII = 0.0;
    if (pI != 0.0) cI = sqrt(gamma * pI / rI);
    if (pII != 0.0) cII = sqrt(gamma * pII / rII);
    const double a = sqrt(rI * (K.g2 * pII + K.g1 * pI) / 2.0);
    const double Uud = (pII - pI) / a;
    const double Urz = -2.0 * cII / K.g1 * (1.0 - pow((pI / pII), K.gm));
    const double Uvk = -2.0 * (cII + cI) / K.g1;
    const double Udf = enI - enII;
    int il = 9, ip = 9, rc = 0;
    double p = 0.0, r = 0.0, te2 = 0.0, te3 = 0.0, en = 0.0, dsl = 0.0, dsp = 0.0, dsc = 0.0;
    if (Udf < Uvk) {
        il = -1;
        ip = -1;
    } else if ((Udf >= Uvk) && (Udf <= Urz)) {
        p = pI * pow(((Udf - Uvk) / (Urz - Uvk)), (1.0 / K.gm));
        il = 0;
        ip = 0;
    } else if ((Udf > Urz) && (Udf <= Uud)) {
        rc = gd_devtwo(K, enI, pI, rI, enII, pII, rII, p);
        il = 1;
        ip = 0;
    } else if (Udf > Uud) {
        rc = gd_newton(K, enI, pI, rI, enII, pII, rII, p);
        il = 1;
        ip = 1;
    }
    if (rc) return rc;
    if (il == 9) return 4;
    if ((il == 1) && (ip == 1)) {  // two shocks
        const double aI = sqrt(rI * (K.g2 / 2.0 * p + K.g1 / 2.0 * pI));
        const double aII = sqrt(rII * (K.g2 / 2.0 * p + K.g1 / 2.0 * pII));
        const double u = (aI * enI + aII * enII + pI - pII) / (aI + aII);
        const double dI = enI - aI / rI;
        const double dII = enII + aII / rII;
        dsl = dI;
        dsp = dII;
        dsc = u;
        if (contact) w = u;
        if (w <= dI) {
            en = enI; p = pI; r = rI; te2 = teI2; te3 = teI3;
        } else if ((w > dI) && (w <= u)) {
            en = u; r = rI * aI / (aI - rI * (enI - u)); te2 = teI2; te3 = teI3;
        } else if ((w > u) && (w < dII)) {
            en = u; r = rII * aII / (aII + rII * (enII - u)); te2 = teII2; te3 = teII3;
        } else if (w >= dII) {
            en = enII; p = pII; r = rII; te2 = teII2; te3 = teII3;
        }
    }
    if ((il == 1) && (ip == 0)) {  // left shock, right rarefaction
        const double aI = sqrt(rI * (K.g2 / 2.0 * p + K.g1 / 2.0 * pI));
        double aII;
        if (fabs(p - pII) < kGodunovEps)
            aII = rII * cII;
        else
            aII = K.gm * rII * cII * (1.0 - p / pII) / (1.0 - pow((p / pII), K.gm));
        const double u = (aI * enI + aII * enII + pI - pII) / (aI + aII);
        const double dI = enI - aI / rI;
        const double dII = enII + cII;
        const double ddII = u + cII - K.g1 * (enII - u) / 2.0;
        dsl = dI;
        dsp = dII;
        dsc = u;
        if (contact) w = u;
        if (w <= dI) {
            en = enI; p = pI; r = rI; te2 = teI2; te3 = teI3;
        }
        if ((w > dI) && (w <= u)) {
            en = u; r = rI * aI / (aI - rI * (enI - u)); te2 = teI2; te3 = teI3;
        }
        if ((w > u) && (w <= ddII)) {
            const double ce = cII - K.g1 / 2.0 * (enII - u);
            en = u; r = K.ga * p / ce / ce; te2 = teII2; te3 = teII3;
        }
        if ((w > ddII) && (w < dII)) {
            const double ce = -K.g1 / K.g2 * (enII - w) + 2.0 / K.g2 * cII;
            en = w - ce; p = pII * pow((ce / cII), (1.0 / K.gm)); r = K.ga * p / ce / ce;
            te2 = teII2; te3 = teII3;
        }
        if (w >= dII) {
            en = enII; p = pII; r = rII; te2 = teII2; te3 = teII3;
        }
    }
    if ((il == 0) && (ip == 0)) {  // two rarefactions
        double aI, aII;
        if (fabs(p - pI) < kGodunovEps)
            aI = rI * cI;
        else
            aI = K.gm * rI * cI * (1.0 - p / pI) / (1.0 - pow((p / pI), K.gm));
        if (fabs(p - pII) < kGodunovEps)
            aII = rII * cII;
        else
            aII = K.gm * rII * cII * (1.0 - p / pII) / (1.0 - pow((p / pII), K.gm));
        const double u = (aI * enI + aII * enII + pI - pII) / (aI + aII);
        const double dI = enI - cI;
        const double ddI = u - cI - K.g1 * (enI - u) / 2.0;
        const double dII = enII + cII;
        const double ddII = u + cII - K.g1 * (enII - u) / 2.0;
        dsl = dI;
        dsp = dII;
        dsc = u;
        if (contact) w = u;
        if (w <= dI) {
            en = enI; p = pI; r = rI; te2 = teI2; te3 = teI3;
        }
        if ((w > dI) && (w < ddI)) {
            const double ce = K.g1 / K.g2 * (enI - w) + 2.0 / K.g2 * cI;
            en = w + ce; p = pI * pow((ce / cI), (1.0 / K.gm)); r = K.ga * p / ce / ce;
            te2 = teI2; te3 = teI3;
        }
        if ((w >= ddI) && (w <= u)) {
            const double ce = cI + K.g1 / 2.0 * (enI - u);
            en = u; r = K.ga * p / ce / ce; te2 = teI2; te3 = teI3;
        }
        if ((w > u) && (w <= ddII)) {
            const double ce = cII - K.g1 / 2.0 * (enII - u);
            en = u; r = K.ga * p / ce / ce; te2 = teII2; te3 = teII3;
        }
        if ((w > ddII) && (w < dII)) {
            const double ce = -K.g1 / K.g2 * (enII - w) + 2.0 / K.g2 * cII;
            en = w - ce; p = pII * pow((ce / cII), (1.0 / K.gm)); r = K.ga * p / ce / ce;
            te2 = teII2; te3 = teII3;
        }
        if (w >= dII) {
            en = enII; p = pII; r = rII; te2 = teII2; te3 = teII3;
        }
    }
    if ((il == -1) && (ip == -1)) {  // vacuum
        const double dI = enI - cI;
        const double ddI = enI + 2.0 / K.g1 * cI;
        const double dII = enII + cII;
        const double ddII = enII - 2.0 / K.g1 * cII;
        dsl = dI;
        dsp = dII;
        dsc = (dI + dII) / 2.0;
        if (contact) w = dsc;
        if (w <= dI) {
            en = enI; p = pI; r = rI; te2 = teI2; te3 = teI3;
        }
        if ((w > dI) && (w < ddI)) {
            const double ce = K.g1 / K.g2 * (enI - w) + 2.0 / K.g2 * cI;
            en = w + ce; p = pI * pow((ce / cI), (1.0 / K.gm)); r = K.ga * p / ce / ce;
            te2 = teI2; te3 = teI3;
        }
        if ((w >= ddI) && (w <= ddII)) {
            en = w; p = 0.0; r = 0.0; te2 = 0.0; te3 = 0.0;
        }
        if ((w > ddII) && (w < dII)) {
            const double ce = -K.g1 / K.g2 * (enII - w) + 2.0 / K.g2 * cII;
            en = w - ce; p = pII * pow((ce / cII), (1.0 / K.gm)); r = K.ga * p / ce / ce;
            te2 = teII2; te3 = teII3;
        }
        if (w >= dII) {
            en = enII; p = pII; r = rII; te2 = teII2; te3 = teII3;
        }
    }
    if (ipiz == 1) {
        en = -en;
        const double dsl1 = dsl, dsp1 = dsp;
        dsl = -dsp1;
        dsp = -dsl1;
        dsc = -dsc;
        w = -w;
    }
    const double uo = al * en + al2 * te2 + al3 * te3;
    const double vo = be * en + be2 * te2 + be3 * te3;
    const double wo = ge * en + ge2 * te2 + ge3 * te3;
    const double eo = p / K.g1 + 0.5 * r * (uo * uo + vo * vo + wo * wo);
    en = al * uo + be * vo + ge * wo;
    if (contact) w = en;
    out[0] = (r * (en - w));
    out[1] = (r * (en - w) * uo + al * p);
    out[2] = (r * (en - w) * vo + be * p);
    out[3] = (r * (en - w) * wo + ge * p);
    out[4] = ((en - w) * eo + en * p);
    ds[0] = dsl;
    ds[1] = dsc;
    ds[2] = dsp;
    return 0;
}


}  // namespace titan

namespace titan {

struct GodunovFlux {
    double q[5];
    double dsl, dsc, dsr;
    int rc;
};

// One HP face with the magnetic pressure folded into p (the preparation of
// Setka_physics.cpp:2378-2388: p += B^2 / (8 pi), B = 0), solved exactly.
// Not inlined: the face kernels call it only for HP faces, and keeping it out
// of line keeps its registers out of the common path. Arguments by value:
// the two face states (rho, u, v, w, p, Bx, By, Bz), Gaussian B.
static __device__ __noinline__ GodunovFlux godunov_hp_face(double n0, double n1, double n2, double w, double r1, double u1,
                                                           double v1, double w1, double p1, double bx1, double by1,
                                                    double bz1, double r2, double u2, double v2, double w2, double p2,
                                                    double bx2, double by2, double bz2, int contact, double gamma) {
    const double nrm[3] = {n0, n1, n2};
    const double q1[5] = {r1, u1, v1, w1, p1 + (bx1 * bx1 + by1 * by1 + bz1 * bz1) / (8.0 * kPi)};
    const double q2[5] = {r2, u2, v2, w2, p2 + (bx2 * bx2 + by2 * by2 + bz2 * bz2) / (8.0 * kPi)};
    GodunovFlux g;
    double ds[3] = {0.0, 0.0, 0.0};
    g.rc = godunov_exact(nrm, w, q1, q2, contact, gamma, g.q, ds);
    g.dsl = ds[0];
    g.dsc = ds[1];
    g.dsr = ds[2];
    return g;
}

}  // namespace titan
