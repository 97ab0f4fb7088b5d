// ============================================================================
// ORACLE — TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of TITAN's plasma time step (`Setka::Go`,
// TITAN/source/Setka_physics.cpp:1484-2278) on flat arrays. Only tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it, and
// only as the checker / the timed CPU baseline — never as the product path.
//
// Parity pin: the Riemann solver below (`o_chlld`) is checked bit-for-bit
// against the reference's own Phys_param::chlld compiled unmodified from the
// reference tree (oracle/Makefile `ref`, tests/test_oracle_ref.py and the
// golden vectors in tests/golden/). The step driver, reconstruction,
// geometry and sources are restatements of the cited reference functions;
// the reference's driver cannot be compiled here (it needs Boost, CGAL,
// Eigen and missing mesh files), so those parts are pinned through the
// reference solver plus invariants (conservation, Test_geometr checks).
//
// Floating point: compiled with -ffp-contract=off so that every expression is
// evaluated in the same order and rounding as the reference's x86-64 build.
// ============================================================================
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// Constants restated from TITAN/source/Header.h:96-104.
const double kPi = 3.14159265358979323846;
const double kCpi4 = 4.0 * kPi;
const double kSpi4 = std::sqrt(kCpi4);
const double kEpsB = 1E-4;
const double kEps = 1E-12;
const double kMeDmp = (1.0 / 1836.15);
// Literal 8*pi used by the energy update, Setka_physics.cpp:1927-1929.
const double kC8Pi = 25.13274122871834590768;

inline double sq(double x) { return x * x; }
inline double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
// std::min / std::max semantics (first argument wins ties and NaN on the left)
inline double mn(double a, double b) { return (b < a) ? b : a; }
inline double mx(double a, double b) { return (a < b) ? b : a; }

}  // namespace

extern "C" {

// ---------------------------------------------------------------------------
// Layout shared with the Python side (tests/oracle_lib.py mirrors it).
// State: SoA [NV][ncell], NV = 10: rho, Vx, Vy, Vz, p, Bx, By, Bz, Q, rho_He.
// H fields (frozen neutral fluids, Bera sources): SoA [5*nh][ncell] in the
// order rho_Hk, Vx_Hk, Vy_Hk, Vz_Hk, p_Hk for k = 1..nh.
// ---------------------------------------------------------------------------
struct OMesh {
    int64_t nnode, ncell, nface;
    const int32_t* cell_nodes;   // ncell*8
    const int32_t* cell_faces;   // ncell*6, the cell's `grans` order
    const int8_t* cell_type;     // ncell, Type_cell (Cell.h:5-11)
    const uint8_t* cell_tvd;     // ncell, Cell::is_TVD
    const int32_t* face_nodes;   // nface*4, nodes around the quad
    const int32_t* face_cells;   // nface*2, cells[0], cells[1] (-1 when absent)
    const int8_t* face_type;     // nface, Type_Gran (Gran.h:5-10)
    const int8_t* face_surf;     // nface, Type_Gran_surf (Gran.h:12-17)
    const int8_t* face_method;   // nface, n_state (policy 0)
    const int32_t* face_bc;      // nface, row of bc_vals for hard faces, else -1
    const double* bc_vals;       // nbc*10, fixed face values (Init_physics)
    const double* node_amp;      // nnode, radial velocity amplitude (ALE), may be null
    const double* node_phase;    // nnode, phase (ALE), may be null
    const int32_t* face_tvd;     // nface*2, Gran::cells_TVD (AA beyond cells[0], BB beyond cells[1]),
                                 // -1 when absent; may be null (no second-order faces)
    // Rays of nodes for the surface-tracking motion (Luch, Luch.h:9-25): node ids
    // from the inner to the outer end, with the radii and the unit direction
    // the ray had when tracking started (oracle_ray_geometry). May be null.
    const int32_t* ray_nodes;    // nray*ray_len
    const double* ray_r0;        // nray*ray_len
    const double* ray_dir;       // nray*3
    int64_t nray, ray_len;
    const int8_t* face_nodt;     // nface, 1: left out of the CFL minimum; may be null
    const double* surf_centre;   // nnode*3, fitted sphere centres of smoothed surface nodes
                                 // (oracle_surface_centres); may be null
    // The A_Luch spacing law for the rays (Luch.cpp:9-152), or null for the
    // fraction rule: M0, M1, M11, M2, M3, M4 (as doubles), R0, R1, R5, da1..da5.
    const double* ray_law;
};

struct OParams {
    double gamma;         // Phys_param::gamma
    double KFL;           // Courant number
    double velosity_inf;  // Phys_param::Velosity_inf (soft-boundary fix-up)
    double omega;         // angular frequency of the prescribed node motion
    double par_a_2, par_n_H_LISM, par_Kn;  // charge exchange (Phys_param.h:111-114)
    double beta_switch;   // policy 1: HLLD where b^2/(2p) > beta_switch, else HLLC
    int32_t move;         // Phys_param::move_setka
    int32_t soft_fixups;  // Outer_Soft fix-ups of Setka_gran_snos.cpp:27-45 (1) or plain copy (0)
    int32_t method_policy;  // 0: face_method array; 1: beta switch per face per step
    int32_t npassive;     // 0 or 2 (Q, rho_He carried as passive scalars)
    int32_t nh;           // number of frozen H fluids feeding the Bera sources (0 = none)
    int32_t TS_hard, contact_hard;
    int32_t tvd;          // Phys_param::TVD: second-order reconstruction on interior faces
    int32_t snos_on_hp;   // Phys_param::Snos_on_HP: second order on HP faces too
    int32_t bn_in_p_on_hp;  // Phys_param::bn_in_p_on_HP: exact gas-dynamic solver on HP faces
    int32_t surface_motion; // node motion by surface tracking (Setka::Culc_Velocity_surface) instead of
                            // the prescribed radial law; needs move and the mesh's rays
    int32_t move_TS, move_HP, move_BS;  // Phys_param::move_TS / move_HP / move_BS
    int32_t null_bn_on_HP;  // Phys_param::null_bn_on_HP
    int32_t pad2;
    double velocity_TS, velocity_HP, velocity_BS;  // Phys_param::velocity_TS / _HP / _BS
    int32_t sglag_TS, sglag_HP, sglag_BS;           // Phys_param::sglag_*: surface smoothing
    int32_t hp_tail;      // HP nodes with x < 0 move along (0, y, z) (Setka_move.cpp:1237-1247)
    double sglag_TS_k_sphere, sglag_HP_k_sphere, sglag_BS_k;
};

struct OStepInfo {
    int64_t steps_done;
    int64_t err_code;     // 0 ok; >0: first failure kind
    int64_t err_index;    // cell or face index of the failure
    int64_t n_rho_floor, n_p_floor;
};

enum { NV = 10 };

// ---------------------------------------------------------------------------
// get_bazis, TITAN/source/Help_funk.cpp:219-232 (Eigen dot / cross / normalized)
// ---------------------------------------------------------------------------
static void o_bazis(const double n[3], double t[3], double m[3]) {
    double a[3] = {1.0, 0.0, 0.0};
    if (std::abs(n[0] * a[0] + n[1] * a[1] + n[2] * a[2]) > 0.9) {
        a[0] = 0.0;
        a[1] = 1.0;
        a[2] = 0.0;
    }
    double c[3] = {a[1] * n[2] - a[2] * n[1], a[2] * n[0] - a[0] * n[2], a[0] * n[1] - a[1] * n[0]};
    double z = c[0] * c[0] + c[1] * c[1] + c[2] * c[2];
    if (z > 0.0) {
        double s = std::sqrt(z);
        t[0] = c[0] / s;
        t[1] = c[1] / s;
        t[2] = c[2] / s;
    } else {
        t[0] = c[0];
        t[1] = c[1];
        t[2] = c[2];
    }
    m[0] = n[1] * t[2] - n[2] * t[1];
    m[1] = n[2] * t[0] - n[0] * t[2];
    m[2] = n[0] * t[1] - n[1] * t[0];
}

// An optional stand-in for o_chlld in the step's face loop: the reference's own
// Phys_param::chlld, compiled unmodified into oracle/_ref behind its C wrapper
// (titan_ref_chlld: the arguments of o_chlld without gamma, which the reference
// holds itself). The CPU-baseline timing installs it so that the Riemann solves,
// most of the step's host time, are the reference's code; results are
// identical (the restatement is bit-exact against it). It reports no status:
// the reference exits on inputs it cannot solve.
using RefRiemann = void (*)(int, const double*, double, const double*, const double*, int, int, int,
                            const double*, const double*, double*, double*, double*, int, int);
static RefRiemann g_ref_riemann = nullptr;

// ---------------------------------------------------------------------------
// Riemann solver family, restating Phys_param::chlld
// (TITAN/source/Phys_param.cpp:882-1878): n_state 0 Lax, 1 HLL, 2 HLLC,
// 3 HLLD, in the frame of a face moving with normal speed w. Returns 0, or a
// nonzero code where the reference prints an error and exits.
// ---------------------------------------------------------------------------
int o_chlld(int n_state, const double* nrm, double w, const double* q1, const double* q2,
            int null_bn, int n_disc, int nk, const double* kl, const double* kr, double* qout,
            double* kout, double* ds, int left_ydar, int contact, double gamma) {
    const double g1 = gamma - 1.0;
    double wv = w;
    const double r1 = q1[0], u1 = q1[1], v1 = q1[2], w1 = q1[3], p1 = q1[4];
    const double bx1 = q1[5] / kSpi4, by1 = q1[6] / kSpi4, bz1 = q1[7] / kSpi4;
    const double r2 = q2[0], u2 = q2[1], v2 = q2[2], w2 = q2[3], p2 = q2[4];
    const double bx2 = q2[5] / kSpi4, by2 = q2[6] / kSpi4, bz2 = q2[7] / kSpi4;
    const double ro = (r2 + r1) / 2.0;
    const double ap = (p2 + p1) / 2.0;

    double n[3] = {nrm[0], nrm[1], nrm[2]}, t[3], m[3];
    o_bazis(n, t, m);

    double vL[3], vR[3], bL[3], bR[3];
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

    // fast magnetosonic speeds (:977-1002)
    const double aaL = bL[0] / std::sqrt(r1);
    const double b2L = dot3(bL, bL);
    const double b21 = b2L / r1;
    const double cL = std::sqrt(gamma * p1 / r1);
    double qp = std::sqrt(b21 + cL * (cL + 2.0 * aaL));
    double qm = std::sqrt(b21 + cL * (cL - 2.0 * aaL));
    const double cfL = (qp + qm) / 2.0;
    const double ptL = p1 + b2L / 2.0;

    const double aaR = bR[0] / std::sqrt(r2);
    const double b2R = dot3(bR, bR);
    const double b22 = b2R / r2;
    const double cR = std::sqrt(gamma * p2 / r2);
    qp = std::sqrt(b22 + cR * (cR + 2.0 * aaR));
    qm = std::sqrt(b22 + cR * (cR - 2.0 * aaR));
    const double cfR = (qp + qm) / 2.0;
    const double ptR = p2 + b2R / 2.0;

    const double aC = (aaL + aaR) / 2.0;
    const double b2o = (b22 + b21) / 2.0;
    const double cC = std::sqrt(gamma * ap / ro);
    qp = std::sqrt(b2o + cC * (cC + 2.0 * aC));
    qm = std::sqrt(b2o + cC * (cC - 2.0 * aC));
    const double cfC = (qp + qm) / 2.0;
    const double vC1 = (vL[0] + vR[0]) / 2.0;

    // wave-speed estimate by n_disc (:1006-1037)
    double SL = 0.0, SR = 0.0;
    if (left_ydar) n_disc = 2;
    if (n_disc == 0) {
        SL = mn(vL[0] - cfL, vR[0] - cfR);
        SR = mx(vL[0] + cfL, vR[0] + cfR);
    } else if (n_disc == 1) {
        SL = mn(vL[0] - cfL, vC1 - cfC);
        SR = mx(vR[0] + cfR, vC1 + cfC);
    } else if (n_disc == 2) {
        const double SL_1 = mn(vL[0] - cfL, vC1 - cfC);
        const double SR_1 = mx(vR[0] + cfR, vC1 + cfC);
        const double SL_2 = mn(vL[0] - cfL, vR[0] - cfR);
        const double SR_2 = mx(vL[0] + cfL, vR[0] + cfR);
        const double oo = 0.6;
        const double oo1 = 1.0 - oo;
        SL = oo * SL_1 + oo1 * SL_2;
        SR = oo * SR_1 + oo1 * SR_2;
    } else if (n_disc == 3) {
        SL = mn(vL[0], vR[0]) - mx(cfL, cfR);
        SR = mx(vL[0], vR[0]) + mx(cfL, cfR);
    }
    ds[2] = SR;
    ds[0] = SL;

    const double suR = SR - vR[0];
    const double suL = SL - vL[0];
    const double SM = (suR * r2 * vR[0] - ptR + ptL - suL * r1 * vL[0]) / (suR * r2 - suL * r1);
    ds[1] = SM;
    if (contact) wv = SM;

    if (n_state == 0) {  // Lax speeds override after dsl/dsr were recorded (:1053-1059)
        const double TR0 = std::fabs(vL[0] + vR[0]) / 2.0 + cfC;
        SR = TR0;
        SL = -TR0;
    }

    const double upt1 = (sq(u1) + sq(v1) + sq(w1)) / 2.0;
    const double sbv1 = u1 * bx1 + v1 * by1 + w1 * bz1;
    const double upt2 = (sq(u2) + sq(v2) + sq(w2)) / 2.0;
    const double sbv2 = u2 * bx2 + v2 * by2 + w2 * bz2;
    const double e1 = p1 / g1 + r1 * upt1 + b2L / 2.0;
    const double e2 = p2 / g1 + r2 * upt2 + b2R / 2.0;

    double FL[8], FR[8], UL[8], UR[8], UZ[8];
    FL[0] = r1 * vL[0];
    FL[1] = r1 * vL[0] * vL[0] + ptL - sq(bL[0]);
    FL[2] = r1 * vL[0] * vL[1] - bL[0] * bL[1];
    FL[3] = r1 * vL[0] * vL[2] - bL[0] * bL[2];
    FL[4] = (e1 + ptL) * vL[0] - bL[0] * sbv1;
    FL[5] = 0.0;
    FL[6] = vL[0] * bL[1] - vL[1] * bL[0];
    FL[7] = vL[0] * bL[2] - vL[2] * bL[0];
    FR[0] = r2 * vR[0];
    FR[1] = r2 * vR[0] * vR[0] + ptR - sq(bR[0]);
    FR[2] = r2 * vR[0] * vR[1] - bR[0] * bR[1];
    FR[3] = r2 * vR[0] * vR[2] - bR[0] * bR[2];
    FR[4] = (e2 + ptR) * vR[0] - bR[0] * sbv2;
    FR[5] = 0.0;
    FR[6] = vR[0] * bR[1] - vR[1] * bR[0];
    FR[7] = vR[0] * bR[2] - vR[2] * bR[0];
    UL[0] = r1;
    UL[4] = e1;
    UR[0] = r2;
    UR[4] = e2;
    for (int i = 0; i < 3; ++i) {
        UL[i + 1] = r1 * vL[i];
        UL[i + 5] = bL[i];
        UR[i + 1] = r2 * vR[i];
        UR[i + 5] = bR[i];
    }
    for (int k = 0; k < 8; ++k) UZ[k] = (SR * UR[k] - SL * UL[k] + FL[k] - FR[k]) / (SR - SL);

    // passive scalars (konvect)
    double FLk[4], FRk[4], UZk[4];
    for (int i = 0; i < nk; ++i) {
        FLk[i] = kl[i] * vL[0];
        FRk[i] = kr[i] * vR[0];
        UZk[i] = (SR * kr[i] - SL * kl[i] + FLk[i] - FRk[i]) / (SR - SL);
    }
    if (null_bn) UZ[5] = 0.0;

    double qv[3], qb[3];
    double SN, wbn;

    if (n_state <= 1) {  // Lax / HLL (:1133-1257)
        double dq[8], FW[8], FWk[4];
        for (int k = 0; k < 8; ++k) dq[k] = UR[k] - UL[k];
        if (left_ydar) wv = SL;
        double TL = SL, TR = SR;
        if (SL > wv || left_ydar) {
            TL = 0.0;
            for (int k = 0; k < 8; ++k) FW[k] = wv * UL[k];
            for (int k = 0; k < nk; ++k) FWk[k] = wv * kl[k];
        } else if (SL <= wv && wv <= SR) {
            for (int k = 0; k < 8; ++k) FW[k] = wv * UZ[k];
            for (int k = 0; k < nk; ++k) FWk[k] = wv * UZk[k];
        } else if (SR < wv) {
            TR = 0.0;
            for (int k = 0; k < 8; ++k) FW[k] = wv * UR[k];
            for (int k = 0; k < nk; ++k) FWk[k] = wv * kr[k];
        } else {
            return 1;
        }
        const double a = TR * TL;
        const double b = TR - TL;
        qout[0] = (TR * FL[0] - TL * FR[0] + a * dq[0]) / b - FW[0];
        qout[4] = (TR * FL[4] - TL * FR[4] + a * dq[4]) / b - FW[4];
        for (int k = 0; k < nk; ++k)
            kout[k] = (TR * FLk[k] - TL * FRk[k] + a * (kr[k] - kl[k])) / b - FWk[k];
        for (int k = 1; k < 4; ++k) qv[k - 1] = (TR * FL[k] - TL * FR[k] + a * dq[k]) / b - FW[k];
        for (int k = 5; k < 8; ++k) qb[k - 5] = (TR * FL[k] - TL * FR[k] + a * dq[k]) / b - FW[k];
        SN = mx(std::fabs(SL), std::fabs(SR));
        if (wv >= SR)
            wbn = wv * bR[0];
        else if (wv <= SL)
            wbn = wv * bL[0];
        else
            wbn = wv * (bL[0] + bR[0]) / 2.0;
    } else if (n_state == 2) {  // HLLC (:1258-1475)
        const double suRm = suR / (SR - SM);
        const double suLm = suL / (SL - SM);
        const double rzR = r2 * suRm;
        const double rzL = r1 * suLm;
        const double ptz =
            (suR * r2 * ptL - suL * r1 * ptR + r1 * r2 * suR * suL * (vR[0] - vL[0])) / (suR * r2 - suL * r1);
        double vzR[3], vzL[3], bzR[3], bzL[3];
        vzR[0] = SM;
        vzL[0] = SM;
        bzR[0] = UZ[5];
        bzL[0] = UZ[5];
        vzR[1] = vR[1] + UZ[5] * (bR[1] - UZ[6]) / suR / r2;
        vzR[2] = vR[2] + UZ[5] * (bR[2] - UZ[7]) / suR / r2;
        vzL[1] = vL[1] + UZ[5] * (bL[1] - UZ[6]) / suL / r1;
        vzL[2] = vL[2] + UZ[5] * (bL[2] - UZ[7]) / suL / r1;
        bzR[1] = UZ[6];
        bzR[2] = UZ[7];
        bzL[1] = bzR[1];
        bzL[2] = bzR[2];
        const double sbvz = (UZ[5] * UZ[1] + UZ[6] * UZ[2] + UZ[7] * UZ[3]) / UZ[0];
        const double ezR = e2 * suRm + (ptz * SM - ptR * vR[0] + UZ[5] * (sbv2 - sbvz)) / (SR - SM);
        const double ezL = e1 * suLm + (ptz * SM - ptL * vL[0] + UZ[5] * (sbv1 - sbvz)) / (SL - SM);
        if (std::fabs(UZ[5]) <= kEpsB) {
            vzR[1] = vR[1];
            vzR[2] = vR[2];
            vzL[1] = vL[1];
            vzL[2] = vL[2];
            bzR[1] = bR[1] * suRm;
            bzR[2] = bR[2] * suRm;
            bzL[1] = bL[1] * suLm;
            bzL[2] = bL[2] * suLm;
        }
        double UZL[8], UZR[8], UZLk[4], UZRk[4];
        for (int k = 0; k < nk; ++k) {
            UZLk[k] = kl[k] * suLm;
            UZRk[k] = kr[k] * suRm;
        }
        UZL[0] = rzL;
        UZL[4] = ezL;
        UZR[0] = rzR;
        UZR[4] = ezR;
        for (int i = 0; i < 3; ++i) {
            UZL[i + 1] = vzL[i] * rzL;
            UZL[i + 5] = bzL[i];
            UZR[i + 1] = vzR[i] * rzR;
            UZR[i + 5] = bzR[i];
        }
        if (left_ydar) wv = SL;
        if (SL >= wv || left_ydar) {
            qout[0] = FL[0] - wv * UL[0];
            qout[4] = FL[4] - wv * UL[4];
            for (int k = 0; k < nk; ++k) kout[k] = FLk[k] - wv * kl[k];
            for (int k = 1; k < 4; ++k) qv[k - 1] = FL[k] - wv * UL[k];
            for (int k = 5; k < 8; ++k) qb[k - 5] = FL[k] - wv * UL[k];
        } else if (SL <= wv && SM >= wv) {
            qout[0] = FL[0] + SL * (rzL - r1) - wv * UZL[0];
            qout[4] = FL[4] + SL * (ezL - e1) - wv * UZL[4];
            for (int k = 0; k < nk; ++k) kout[k] = FLk[k] + SL * (UZLk[k] - kl[k]) - wv * UZLk[k];
            for (int k = 1; k < 4; ++k) qv[k - 1] = FL[k] + SL * (UZL[k] - UL[k]) - wv * UZL[k];
            for (int k = 5; k < 8; ++k) qb[k - 5] = FL[k] + SL * (UZL[k] - UL[k]) - wv * UZL[k];
        } else if (SM <= wv && SR > wv) {
            qout[0] = FR[0] + SR * (rzR - r2) - wv * UZR[0];
            qout[4] = FR[4] + SR * (ezR - e2) - wv * UZR[4];
            for (int k = 0; k < nk; ++k) kout[k] = FRk[k] + SR * (UZRk[k] - kr[k]) - wv * UZRk[k];
            for (int k = 1; k < 4; ++k) qv[k - 1] = FR[k] + SR * (UZR[k] - UR[k]) - wv * UZR[k];
            for (int k = 5; k < 8; ++k) qb[k - 5] = FR[k] + SR * (UZR[k] - UR[k]) - wv * UZR[k];
        } else if (SR <= wv) {
            qout[0] = FR[0] - wv * UR[0];
            qout[4] = FR[4] - wv * UR[4];
            for (int k = 0; k < nk; ++k) kout[k] = FRk[k] - wv * kr[k];
            for (int k = 1; k < 4; ++k) qv[k - 1] = FR[k] - wv * UR[k];
            for (int k = 5; k < 8; ++k) qb[k - 5] = FR[k] - wv * UR[k];
        } else {
            return 2;
        }
        SN = mx(std::fabs(SL), std::fabs(SR));
        if (wv > SR)
            wbn = wv * bR[0];
        else if (wv < SL)
            wbn = wv * bL[0];
        else
            wbn = wv * (bL[0] + bR[0]) / 2.0;
    } else if (n_state == 3) {  // HLLD (:1476-1870)
        const double ptz =
            (suR * r2 * ptL - suL * r1 * ptR + r1 * r2 * suR * suL * (vR[0] - vL[0])) / (suR * r2 - suL * r1);
        double vzL[3], vzR[3], vzzL[3], vzzR[3], bzL[3], bzR[3], bzzL[3], bzzR[3];
        vzL[0] = SM;
        vzR[0] = SM;
        vzzL[0] = SM;
        vzzR[0] = SM;
        const double suRm = suR / (SR - SM);
        const double suLm = suL / (SL - SM);
        const double rzR = r2 * suRm;
        const double rzL = r1 * suLm;
        double qzL[4], qzR[4];
        for (int k = 0; k < nk; ++k) {
            qzL[k] = kl[k] * suLm;
            qzR[k] = kr[k] * suRm;
        }
        const double bn = UZ[5];
        const double bn2 = bn * bn;
        bzL[0] = bn;
        bzR[0] = bn;
        bzzL[0] = bn;
        bzzR[0] = bn;
        double tvR, tbR, tvL, tbL;
        const double ttR = r2 * suR * (SR - SM) - bn2;
        if (std::fabs(ttR) < 0.000000001) {
            tvR = 0.0;
            tbR = 0.0;
        } else {
            tvR = (SM - vR[0]) / ttR;
            tbR = (r2 * suR * suR - bn2) / ttR;
        }
        const double ttL = r1 * suL * (SL - SM) - bn2;
        if (std::fabs(ttL) < 0.000000001) {
            tvL = 0.0;
            tbL = 0.0;
        } else {
            tvL = (SM - vL[0]) / ttL;
            tbL = (r1 * suL * suL - bn2) / ttL;
        }
        vzL[1] = vL[1] - bn * bL[1] * tvL;
        vzL[2] = vL[2] - bn * bL[2] * tvL;
        vzR[1] = vR[1] - bn * bR[1] * tvR;
        vzR[2] = vR[2] - bn * bR[2] * tvR;
        bzL[1] = bL[1] * tbL;
        bzL[2] = bL[2] * tbL;
        bzR[1] = bR[1] * tbR;
        bzR[2] = bR[2] * tbR;
        const double sbvL = bzL[0] * vzL[0] + bzL[1] * vzL[1] + bzL[2] * vzL[2];
        const double sbvR = bzR[0] * vzR[0] + bzR[1] * vzR[1] + bzR[2] * vzR[2];
        const double ezR = e2 * suRm + (ptz * SM - ptR * vR[0] + bn * (sbv2 - sbvR)) / (SR - SM);
        const double ezL = e1 * suLm + (ptz * SM - ptL * vL[0] + bn * (sbv1 - sbvL)) / (SL - SM);
        const double rzRs = std::sqrt(rzR);
        const double rzLs = std::sqrt(rzL);
        const double rzss = rzRs + rzLs;
        const double rzps = rzRs * rzLs;
        double SZL = SM - std::fabs(bn) / rzLs;
        double SZR = SM + std::fabs(bn) / rzRs;
        double sbn;
        int ibn;
        if (std::fabs(bn) > kEpsB) {
            sbn = std::fabs(bn) / bn;
            ibn = 1;
        } else {
            sbn = 0.0;
            ibn = 0;
            SZL = SM;
            SZR = SM;
        }
        vzzL[1] = (rzLs * vzL[1] + rzRs * vzR[1] + sbn * (bzR[1] - bzL[1])) / rzss;
        vzzL[2] = (rzLs * vzL[2] + rzRs * vzR[2] + sbn * (bzR[2] - bzL[2])) / rzss;
        vzzR[1] = vzzL[1];
        vzzR[2] = vzzL[2];
        bzzL[1] = (rzLs * bzR[1] + rzRs * bzL[1] + sbn * rzps * (vzR[1] - vzL[1])) / rzss;
        bzzL[2] = (rzLs * bzR[2] + rzRs * bzL[2] + sbn * rzps * (vzR[2] - vzL[2])) / rzss;
        bzzR[1] = bzzL[1];
        bzzR[2] = bzzL[2];
        const double sbzz = bzzL[0] * vzzL[0] + bzzL[1] * vzzL[1] + bzzL[2] * vzzL[2];
        const double ezzR = ezR + rzRs * sbn * (sbvR - sbzz);
        const double ezzL = ezL - rzLs * sbn * (sbvL - sbzz);
        double UZL[8], UZR[8], UZZL[8], UZZR[8];
        UZL[0] = rzL;
        UZL[4] = ezL;
        UZR[0] = rzR;
        UZR[4] = ezR;
        UZZL[0] = rzL;
        UZZL[4] = ezzL;
        UZZR[0] = rzR;
        UZZR[4] = ezzR;
        for (int i = 0; i < 3; ++i) {
            UZL[i + 1] = vzL[i] * rzL;
            UZL[i + 5] = bzL[i];
            UZR[i + 1] = vzR[i] * rzR;
            UZR[i + 5] = bzR[i];
            UZZL[i + 1] = vzzL[i] * rzL;
            UZZL[i + 5] = bzzL[i];
            UZZR[i + 1] = vzzR[i] * rzR;
            UZZR[i + 5] = bzzR[i];
        }
        int j_ccs = -1;
        if (left_ydar) wv = SL;
        if (SL >= wv || left_ydar) {  // zone 1
            qout[0] = FL[0] - wv * UL[0];
            qout[4] = FL[4] - wv * UL[4];
            for (int k = 1; k < 4; ++k) qv[k - 1] = FL[k] - wv * UL[k];
            for (int k = 5; k < 8; ++k) qb[k - 5] = FL[k] - wv * UL[k];
            for (int k = 0; k < nk; ++k) kout[k] = FLk[k] - wv * kl[k];
            j_ccs = 1;
        } else if (SL <= wv && SZL >= wv) {  // zone 2
            for (int k : {0, 4}) qout[k] = FL[k] + SL * (UZL[k] - UL[k]) - wv * UZL[k];
            for (int k = 0; k < nk; ++k) kout[k] = FLk[k] + SL * (qzL[k] - kl[k]) - wv * qzL[k];
            for (int k = 1; k < 4; ++k) qv[k - 1] = FL[k] + SL * (UZL[k] - UL[k]) - wv * UZL[k];
            for (int k = 5; k < 8; ++k) qb[k - 5] = FL[k] + SL * (UZL[k] - UL[k]) - wv * UZL[k];
            j_ccs = 2;
        }
        if (ibn == 1) {
            if (SZL <= wv && SM >= wv) {  // zone 3
                for (int k : {0, 4})
                    qout[k] = FL[k] + SZL * (UZZL[k] - UZL[k]) + SL * (UZL[k] - UL[k]) - wv * UZZL[k];
                for (int k = 0; k < nk; ++k)
                    kout[k] = FLk[k] + SZL * (qzL[k] - qzL[k]) + SL * (qzL[k] - kl[k]) - wv * qzL[k];
                for (int k = 1; k < 4; ++k)
                    qv[k - 1] = FL[k] + SZL * (UZZL[k] - UZL[k]) + SL * (UZL[k] - UL[k]) - wv * UZZL[k];
                for (int k = 5; k < 8; ++k)
                    qb[k - 5] = FL[k] + SZL * (UZZL[k] - UZL[k]) + SL * (UZL[k] - UL[k]) - wv * UZZL[k];
                j_ccs = 3;
            } else if (SM <= wv && SZR >= wv) {  // zone 4
                for (int k : {0, 4})
                    qout[k] = FR[k] + SZR * (UZZR[k] - UZR[k]) + SR * (UZR[k] - UR[k]) - wv * UZZR[k];
                for (int k = 0; k < nk; ++k)
                    kout[k] = FRk[k] + SZR * (qzR[k] - qzR[k]) + SR * (qzR[k] - kr[k]) - wv * qzR[k];
                for (int k = 1; k < 4; ++k)
                    qv[k - 1] = FR[k] + SZR * (UZZR[k] - UZR[k]) + SR * (UZR[k] - UR[k]) - wv * UZZR[k];
                for (int k = 5; k < 8; ++k)
                    qb[k - 5] = FR[k] + SZR * (UZZR[k] - UZR[k]) + SR * (UZR[k] - UR[k]) - wv * UZZR[k];
                j_ccs = 4;
            }
        }
        if (SZR <= wv && SR >= wv) {  // zone 5
            for (int k : {0, 4}) qout[k] = FR[k] + SR * (UZR[k] - UR[k]) - wv * UZR[k];
            for (int k = 0; k < nk; ++k) kout[k] = FRk[k] + SR * (qzR[k] - kr[k]) - wv * qzR[k];
            for (int k = 1; k < 4; ++k) qv[k - 1] = FR[k] + SR * (UZR[k] - UR[k]) - wv * UZR[k];
            for (int k = 5; k < 8; ++k) qb[k - 5] = FR[k] + SR * (UZR[k] - UR[k]) - wv * UZR[k];
            j_ccs = 5;
        } else if (SR <= wv) {  // zone 6
            qout[0] = FR[0] - wv * UR[0];
            qout[4] = FR[4] - wv * UR[4];
            for (int k = 0; k < nk; ++k) kout[k] = FRk[k] - wv * kr[k];
            for (int k = 1; k < 4; ++k) qv[k - 1] = FR[k] - wv * UR[k];
            for (int k = 5; k < 8; ++k) qb[k - 5] = FR[k] - wv * UR[k];
            j_ccs = 6;
        }
        if (j_ccs == -1) return 3;
        SN = mx(std::fabs(SL), std::fabs(SR));
        if (wv > SR)
            wbn = wv * bR[0];
        else if (wv < SL)
            wbn = wv * bL[0];
        else
            wbn = wv * (bL[0] + bR[0]) / 2.0;
    } else {
        return 4;
    }
    // normal-B flux (Powell form) and rotation back with the sqrt(4 pi) rescale
    qb[0] = -SN * (bR[0] - bL[0]) - wbn;
    if (null_bn) qb[0] = 0.0;
    for (int i = 0; i < 3; ++i) {
        qout[i + 1] = n[i] * qv[0] + t[i] * qv[1] + m[i] * qv[2];
        qout[i + 5] = n[i] * qb[0] + t[i] * qb[1] + m[i] * qb[2];
        qout[i + 5] = kSpi4 * qout[i + 5];
    }
    return 0;
}

// ---------------------------------------------------------------------------
// Geometry, restating Setka::Calculating_measure (Setka.cpp:2465-2502):
// cell centres (Cell.cpp:909-930) -> face centre / area / oriented normal
// (Gran.cpp:112-218) -> cell volume, method 1 (Cell.cpp:958-1001).
// Outputs: cc[3*ncell], vol[ncell], fc[3*nface], fn[3*nface], fa[nface].
// ---------------------------------------------------------------------------
static double tri_area(const double* a, const double* b, const double* c) {
    const double v1x = b[0] - a[0], v1y = b[1] - a[1], v1z = b[2] - a[2];
    const double v2x = c[0] - a[0], v2y = c[1] - a[1], v2z = c[2] - a[2];
    const double cx = v1y * v2z - v1z * v2y;
    const double cy = v1z * v2x - v1x * v2z;
    const double cz = v1x * v2y - v1y * v2x;
    return 0.5 * std::sqrt(cx * cx + cy * cy + cz * cz);
}

static double tet_vol(const double* a, const double* b, const double* c, const double* d) {
    const double abx = b[0] - a[0], aby = b[1] - a[1], abz = b[2] - a[2];
    const double acx = c[0] - a[0], acy = c[1] - a[1], acz = c[2] - a[2];
    const double adx = d[0] - a[0], ady = d[1] - a[1], adz = d[2] - a[2];
    const double cx = aby * acz - abz * acy;
    const double cy = abz * acx - abx * acz;
    const double cz = abx * acy - aby * acx;
    const double dp = cx * adx + cy * ady + cz * adz;
    return std::abs(dp) / 6.0;
}

void oracle_geometry(const OMesh* M, const double* xyz, double* cc, double* vol, double* fc,
                     double* fn, double* fa) {
    const int64_t nc = M->ncell, nf = M->nface;
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < nc; ++c) {
        double x = 0.0, y = 0.0, z = 0.0;
        for (int k = 0; k < 8; ++k) {
            const double* p = xyz + 3 * (int64_t)M->cell_nodes[8 * c + k];
            x += p[0];
            y += p[1];
            z += p[2];
        }
        cc[3 * c + 0] = x / 8;
        cc[3 * c + 1] = y / 8;
        cc[3 * c + 2] = z / 8;
    }
#pragma omp parallel for schedule(static)
    for (int64_t f = 0; f < nf; ++f) {
        const double* P[4];
        for (int k = 0; k < 4; ++k) P[k] = xyz + 3 * (int64_t)M->face_nodes[4 * f + k];
        double xc = 0.0, yc = 0.0, zc = 0.0;
        for (int k = 0; k < 4; ++k) {
            xc += P[k][0];
            yc += P[k][1];
            zc += P[k][2];
        }
        xc /= 4;
        yc /= 4;
        zc /= 4;
        fc[3 * f + 0] = xc;
        fc[3 * f + 1] = yc;
        fc[3 * f + 2] = zc;
        double S = 0.0;
        S += tri_area(P[0], P[1], P[2]);
        S += tri_area(P[0], P[3], P[2]);
        fa[f] = S;
        const double x1 = (P[0][0] + P[1][0]) / 2.0, y1 = (P[0][1] + P[1][1]) / 2.0, z1 = (P[0][2] + P[1][2]) / 2.0;
        const double x2 = (P[1][0] + P[2][0]) / 2.0, y2 = (P[1][1] + P[2][1]) / 2.0, z2 = (P[1][2] + P[2][2]) / 2.0;
        const double x3 = (P[2][0] + P[3][0]) / 2.0, y3 = (P[2][1] + P[3][1]) / 2.0, z3 = (P[2][2] + P[3][2]) / 2.0;
        const double ax = x2 - x1, ay = y2 - y1, az = z2 - z1;
        const double bx = x3 - x1, by = y3 - y1, bz = z3 - z1;
        double n1 = ay * bz - az * by;
        double n2 = az * bx - ax * bz;
        double n3 = ax * by - ay * bx;
        const double nn = std::sqrt(n1 * n1 + n2 * n2 + n3 * n3);
        n1 /= nn;
        n2 /= nn;
        n3 /= nn;
        const double* c0 = cc + 3 * (int64_t)M->face_cells[2 * f];
        if (n1 * (c0[0] - xc) + n2 * (c0[1] - yc) + n3 * (c0[2] - zc) > 0.0) {
            n1 = -n1;
            n2 = -n2;
            n3 = -n3;
        }
        fn[3 * f + 0] = n1;
        fn[3 * f + 1] = n2;
        fn[3 * f + 2] = n3;
    }
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < nc; ++c) {
        double V = 0.0;
        const double* C = cc + 3 * c;
        for (int s = 0; s < 6; ++s) {
            const int32_t* fnd = M->face_nodes + 4 * (int64_t)M->cell_faces[6 * c + s];
            const double* P0 = xyz + 3 * (int64_t)fnd[0];
            const double* P1 = xyz + 3 * (int64_t)fnd[1];
            const double* P2 = xyz + 3 * (int64_t)fnd[2];
            const double* P3 = xyz + 3 * (int64_t)fnd[3];
            V += tet_vol(C, P0, P1, P2);
            V += tet_vol(C, P0, P3, P2);
        }
        vol[c] = V;
    }
}

// ---------------------------------------------------------------------------
// Spherical <-> Cartesian vector helpers, TITAN/source/Help_funk.cpp:75-135.
// ---------------------------------------------------------------------------
static double o_polar_angle(double x, double y) {
    if (std::fabs(x) + std::fabs(y) < 0.000001) return 0.0;
    if (x < 0) return std::atan(y / x) + 1.0 * kPi;
    if (x > 0 && y >= 0) return std::atan(y / x);
    if (x > 0 && y < 0) return std::atan(y / x) + 2.0 * kPi;
    if (y > 0 && x >= 0 && x <= 0) return kPi / 2.0;
    if (y < 0 && x >= 0 && x <= 0) return 3.0 * kPi / 2.0;
    return 0.0;
}

static void o_spherical(double z, double x, double y, double Vz, double Vx, double Vy, double& Vr,
                        double& Vphi, double& Vtheta) {
    const double r = std::sqrt(x * x + y * y + z * z);
    const double th = std::acos(z / r);
    const double ph = o_polar_angle(x, y);
    Vr = Vx * std::sin(th) * std::cos(ph) + Vy * std::sin(th) * std::sin(ph) + Vz * std::cos(th);
    Vtheta = Vx * std::cos(th) * std::cos(ph) + Vy * std::cos(th) * std::sin(ph) - Vz * std::sin(th);
    Vphi = -Vx * std::sin(ph) + Vy * std::cos(ph);
}

static void o_cartesian(double z, double x, double y, double Vr, double Vphi, double Vtheta, double& Vz,
                        double& Vx, double& Vy) {
    const double r = std::sqrt(x * x + y * y + z * z);
    const double th = std::acos(z / r);
    const double ph = o_polar_angle(x, y);
    Vx = Vr * std::sin(th) * std::cos(ph) + Vtheta * std::cos(th) * std::cos(ph) - Vphi * std::sin(ph);
    Vy = Vr * std::sin(th) * std::sin(ph) + Vtheta * std::cos(th) * std::sin(ph) + Vphi * std::cos(ph);
    Vz = Vr * std::cos(th) - Vtheta * std::sin(th);
}

// First-order interior reconstruction of one side, Setka_gran_snos.cpp:737-907
// (cells[0]) and :909-1069 (cells[1]): Zone_1 cells are scaled radially from
// the cell centre to the face centre; other cells are copied.
static void o_snos_side(const double* st, int64_t nc, int64_t c, int ctype, const double* cc, const double* G,
                        double gamma, double* out) {
    for (int k = 0; k < NV; ++k) out[k] = st[k * nc + c];
    if (ctype != 1) return;
    const double* Ac = cc + 3 * c;
    const double r1 = std::sqrt(Ac[0] * Ac[0] + Ac[1] * Ac[1] + Ac[2] * Ac[2]);
    const double rr = std::sqrt(G[0] * G[0] + G[1] * G[1] + G[2] * G[2]);
    const double the1 = std::acos(G[2] / rr);
    for (int ik = 0; ik < 2; ++ik) {  // ik 0: velocity, 1: magnetic field
        const int i1 = ik == 0 ? 1 : 5;
        const double AX = st[(i1 + 0) * nc + c], AY = st[(i1 + 1) * nc + c], AZ = st[(i1 + 2) * nc + c];
        double VA0, VA1, VA2;
        if (the1 > kPi / 9 && the1 < 8 * kPi / 9) {
            o_spherical(Ac[2], Ac[0], Ac[1], AZ, AX, AY, VA0, VA1, VA2);
            if (ik == 1) {
                VA0 = VA0 * (sq(r1 / rr));
                VA1 = VA1 * ((r1) / (rr));
                VA2 = VA2 * ((r1) / (rr));
            }
            o_cartesian(G[2], G[0], G[1], VA0, VA1, VA2, out[i1 + 2], out[i1 + 0], out[i1 + 1]);
        } else {
            o_spherical(Ac[0], Ac[1], Ac[2], AX, AY, AZ, VA0, VA1, VA2);
            if (ik == 1) {
                VA0 = VA0 * (sq(r1 / rr));
                VA1 = VA1 * ((r1) / (rr));
                VA2 = VA2 * ((r1) / (rr));
            }
            o_cartesian(G[0], G[1], G[2], VA0, VA1, VA2, out[i1 + 0], out[i1 + 1], out[i1 + 2]);
        }
    }
    out[0] = st[0 * nc + c] * sq(r1) / sq(rr);
    out[8] = st[8 * nc + c] * sq(r1) / sq(rr);
    out[9] = st[9 * nc + c] * sq(r1) / sq(rr);
    out[4] = st[4 * nc + c] * std::pow(r1, 2.0 * gamma) / std::pow(rr, 2.0 * gamma);
}

// ---------------------------------------------------------------------------
// Exact gas-dynamic Godunov solver of HP faces with bn_in_p_on_HP,
// Phys_param::Godunov_Solver_Alexashov (Phys_param.cpp:1938-2385) with its
// Newton (:2387-2442), bisection (:2444-2519) and pressure-function (:2521-2536)
// helpers. The reference's macros (Phys_param.cpp:3-11: ga = gamma, g1 =
// ga - 1, g2 = ga + 1, gp = (g2/ga)/2, gm = (g1/ga)/2, gga = ga) are
// parenthesised, so their values are formed once here. Where the reference
// exits (negative pressure in Newton, 1100 iterations without convergence)
// this returns 1 / 2 / 3; 4 where no wave pattern applies (NaN input).
// q1, q2: rho, u, v, w, p; out: 5 fluxes; ds: dsl, dsc, dsr.
// ---------------------------------------------------------------------------
namespace {
struct GodunovK {
    double ga, g1, g2, gp, gm;
    explicit GodunovK(double gamma)
        : ga(gamma), g1(gamma - 1.0), g2(gamma + 1.0), gp(((gamma + 1.0) / gamma) / 2.0),
          gm(((gamma - 1.0) / gamma) / 2.0) {}
};

double o_lev(const GodunovK& K, double enI, double pI, double rI, double enII, double pII, double rII, double uuu) {
    const double cI = std::sqrt(K.ga * pI / rI);
    const double cII = std::sqrt(K.ga * pII / rII);
    const double fI = (uuu - pI) / (rI * cI * std::sqrt(K.gp * uuu / pI + K.gm));
    const double fII = 2.0 / K.g1 * cII * (std::pow((uuu / pII), K.gm) - 1.0);
    const double f1 = fI + fII;
    const double f2 = enI - enII;
    return f1 - f2;
}

int o_newton(const GodunovK& K, double enI, double pI, double rI, double enII, double pII, double rII, double& p) {
    const double cI = std::sqrt(K.ga * pI / rI);
    const double cII = std::sqrt(K.ga * pII / rII);
    double pn = pI * rII * cII + pII * rI * cI + (enI - enII) * rI * cI * rII * cII;
    pn = pn / (rI * cI + rII * cII);
    const double pee = pn;
    int kiter = 0;
    while (true) {
        p = pn;
        if (p <= 0.0) return 1;
        kiter = kiter + 1;
        const double fI = (p - pI) / (rI * cI * std::sqrt(K.gp * p / pI + K.gm));
        double fIs = (K.ga + 1.0) * p / pI + (3.0 * K.ga - 1.0);
        fIs = fIs / (4.0 * K.ga * rI * cI * std::pow((K.gp * p / pI + K.gm), (3.0 / 2.0)));
        const double fII = (p - pII) / (rII * cII * std::sqrt(K.gp * p / pII + K.gm));
        double fIIs = (K.ga + 1.0) * p / pII + (3.0 * K.ga - 1.0);
        fIIs = fIIs / (4.0 * K.ga * rII * cII * std::pow((K.gp * p / pII + K.gm), (3.0 / 2.0)));
        if (kiter == 1100) return 2;
        pn = p - (fI + fII - (enI - enII)) / (fIs + fIIs);
        if (!(std::fabs(pn / pee - p / pee) >= kEps)) break;
    }
    p = pn;
    return 0;
}

int o_devtwo(const GodunovK& K, double enI, double pI, double rI, double enII, double pII, double rII, double& p) {
    const double epsil = 10e-10;
    double kl = pI, kp = pII;
    double ksi = o_lev(K, enI, pI, rI, enII, pII, rII, kl);
    double ksir = o_lev(K, enI, pI, rI, enII, pII, rII, kp);
    if (std::fabs(ksi) <= epsil) {
        p = kl;
        return 0;
    }
    if (std::fabs(ksir) <= epsil) {
        p = kp;
        return 0;
    }
    int kpizd = 0;
    while (true) {
        kpizd = kpizd + 1;
        if (kpizd == 1100) return 3;
        const double kc = (kl + kp) / 2.0;
        const double ksit = o_lev(K, enI, pI, rI, enII, pII, rII, kc);
        if (std::fabs(ksit) <= epsil) {
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
}  // namespace

int o_godunov(const double* nrm, double w, const double* q1, const double* q2, int contact, double gamma,
              double* out, double* ds) {
    const GodunovK K(gamma);
    const double al = nrm[0], be = nrm[1], ge = nrm[2];
    double t[3], m[3];
    o_bazis(nrm, t, m);
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
    if (pI != 0.0) cI = std::sqrt(gamma * pI / rI);
    if (pII != 0.0) cII = std::sqrt(gamma * pII / rII);
    const double a = std::sqrt(rI * (K.g2 * pII + K.g1 * pI) / 2.0);
    const double Uud = (pII - pI) / a;
    const double Urz = -2.0 * cII / K.g1 * (1.0 - std::pow((pI / pII), K.gm));
    const double Uvk = -2.0 * (cII + cI) / K.g1;
    const double Udf = enI - enII;
    int il = 9, ip = 9, rc = 0;
    double p = 0.0, r = 0.0, te2 = 0.0, te3 = 0.0, en = 0.0, dsl = 0.0, dsp = 0.0, dsc = 0.0;
    if (Udf < Uvk) {
        il = -1;
        ip = -1;
    } else if ((Udf >= Uvk) && (Udf <= Urz)) {
        p = pI * std::pow(((Udf - Uvk) / (Urz - Uvk)), (1.0 / K.gm));
        il = 0;
        ip = 0;
    } else if ((Udf > Urz) && (Udf <= Uud)) {
        rc = o_devtwo(K, enI, pI, rI, enII, pII, rII, p);
        il = 1;
        ip = 0;
    } else if (Udf > Uud) {
        rc = o_newton(K, enI, pI, rI, enII, pII, rII, p);
        il = 1;
        ip = 1;
    }
    if (rc) return rc;
    if (il == 9) return 4;
    if ((il == 1) && (ip == 1)) {  // two shocks
        const double aI = std::sqrt(rI * (K.g2 / 2.0 * p + K.g1 / 2.0 * pI));
        const double aII = std::sqrt(rII * (K.g2 / 2.0 * p + K.g1 / 2.0 * pII));
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
        const double aI = std::sqrt(rI * (K.g2 / 2.0 * p + K.g1 / 2.0 * pI));
        double aII;
        if (std::fabs(p - pII) < kEps)
            aII = rII * cII;
        else
            aII = K.gm * rII * cII * (1.0 - p / pII) / (1.0 - std::pow((p / pII), K.gm));
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
            en = w - ce; p = pII * std::pow((ce / cII), (1.0 / K.gm)); r = K.ga * p / ce / ce;
            te2 = teII2; te3 = teII3;
        }
        if (w >= dII) {
            en = enII; p = pII; r = rII; te2 = teII2; te3 = teII3;
        }
    }
    if ((il == 0) && (ip == 0)) {  // two rarefactions
        double aI, aII;
        if (std::fabs(p - pI) < kEps)
            aI = rI * cI;
        else
            aI = K.gm * rI * cI * (1.0 - p / pI) / (1.0 - std::pow((p / pI), K.gm));
        if (std::fabs(p - pII) < kEps)
            aII = rII * cII;
        else
            aII = K.gm * rII * cII * (1.0 - p / pII) / (1.0 - std::pow((p / pII), K.gm));
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
            en = w + ce; p = pI * std::pow((ce / cI), (1.0 / K.gm)); r = K.ga * p / ce / ce;
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
            en = w - ce; p = pII * std::pow((ce / cII), (1.0 / K.gm)); r = K.ga * p / ce / ce;
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
            en = w + ce; p = pI * std::pow((ce / cI), (1.0 / K.gm)); r = K.ga * p / ce / ce;
            te2 = teI2; te3 = teI3;
        }
        if ((w >= ddI) && (w <= ddII)) {
            en = w; p = 0.0; r = 0.0; te2 = 0.0; te3 = 0.0;
        }
        if ((w > ddII) && (w < dII)) {
            const double ce = -K.g1 / K.g2 * (enII - w) + 2.0 / K.g2 * cII;
            en = w - ce; p = pII * std::pow((ce / cII), (1.0 / K.gm)); r = K.ga * p / ce / ce;
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

// ---------------------------------------------------------------------------
// Second-order (TVD) reconstruction, Setka_gran_snos.cpp:188-735.
// Cells on the line AA - A -|- B - BB (AA beyond cells[0], BB beyond
// cells[1], Init_TVD) at coordinates -dd1-d1, -d1, 0 (face centre), d2,
// d2+dd2. linear (Help_funk.cpp:55-63): minmod of the two slopes through
// the middle point; linear2 (:65-70): the line through two points; both
// evaluated at the face (y = 0).
// ---------------------------------------------------------------------------
static int o_signum(double x) { return x > 0.00000001 ? 1 : (x < -0.00000001 ? -1 : 0); }

static double o_minmod(double x, double y) {
    if (o_signum(x) + o_signum(y) == 0) return 0.0;
    return ((o_signum(x) + o_signum(y)) / 2.0) * mn(std::fabs(x), std::fabs(y));
}

static double o_lin3(double x1, double t1, double x2, double t2, double x3, double t3) {
    const double y = 0.0;
    const double d = o_minmod((t1 - t2) / (x1 - x2), (t2 - t3) / (x2 - x3));
    return (d * (y - x2) + t2);
}

static double o_lin2(double x1, double t1, double x2, double t2) {
    const double y = 0.0;
    const double d = (t1 - t2) / (x1 - x2);
    return (d * (y - x2) + t2);
}

static inline double o_norm3(const double* a) { return std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); }

// Face states L, R of an interior face on the second-order branch.
// c[0..3] = AA, A, B, BB; ctype their Type_cell.
static void o_snos_tvd(const double* st, int64_t nc, const int64_t c[4], const int ct[4], const double* cc,
                       const double* G, double gamma, int npassive, double* L, double* R) {
    const double *AAc = cc + 3 * c[0], *Ac = cc + 3 * c[1], *Bc = cc + 3 * c[2], *BBc = cc + 3 * c[3];
    double v[3];
    for (int j = 0; j < 3; ++j) v[j] = Ac[j] - G[j];
    const double d1 = o_norm3(v);
    for (int j = 0; j < 3; ++j) v[j] = Bc[j] - G[j];
    const double d2 = o_norm3(v);
    for (int j = 0; j < 3; ++j) v[j] = Ac[j] - AAc[j];
    const double dd1 = o_norm3(v);
    for (int j = 0; j < 3; ++j) v[j] = Bc[j] - BBc[j];
    const double dd2 = o_norm3(v);
    const double xAA = -dd1 - d1, xA = -d1, xB = d2, xBB = d2 + dd2;
    auto S = [&](int k, int i) { return st[(int64_t)k * nc + c[i]]; };
    const int a0 = ct[0], a1 = ct[1], b1 = ct[2], b0 = ct[3];
    const bool z1111 = a0 == 1 && a1 == 1 && b1 == 1 && b0 == 1;
    const bool z1112 = a0 == 1 && a1 == 1 && b1 == 1 && b0 == 2;
    const bool z1122 = a0 == 1 && a1 == 1 && b1 == 2 && b0 == 2;
    const bool z1222 = a0 == 1 && a1 == 2 && b1 == 2 && b0 == 2;
    if (z1111 || z1112 || z1122) {
        const double r3 = o_norm3(AAc), r1 = o_norm3(Ac), rr = o_norm3(G), r2 = o_norm3(Bc), r4 = o_norm3(BBc);
        const double the1 = std::acos(G[2] / rr);
        const bool band = the1 > kPi / 9 && the1 < 8 * kPi / 9;
        // spherical components (Vr, Vphi, Vtheta) of a vector field of cell i,
        // in the frame the band test selects (Setka_gran_snos.cpp:241-254 / :301-315)
        auto sph = [&](int i, int k0, double* out) {
            const double* X = cc + 3 * c[i];
            const double vx = S(k0, i), vy = S(k0 + 1, i), vz = S(k0 + 2, i);
            if (band)
                o_spherical(X[2], X[0], X[1], vz, vx, vy, out[0], out[1], out[2]);
            else
                o_spherical(X[0], X[1], X[2], vx, vy, vz, out[0], out[1], out[2]);
        };
        auto cart = [&](const double* Vs, double* side, int k0) {
            if (band)
                o_cartesian(G[2], G[0], G[1], Vs[0], Vs[1], Vs[2], side[k0 + 2], side[k0], side[k0 + 1]);
            else
                o_cartesian(G[0], G[1], G[2], Vs[0], Vs[1], Vs[2], side[k0], side[k0 + 1], side[k0 + 2]);
        };
        for (int ik = 0; ik < 2; ++ik) {
            const int k0 = ik == 0 ? 1 : 5;
            double VAA[3], VA[3], VB[3], VBB[3], Vl[3], Vr[3];
            sph(0, k0, VAA);
            sph(1, k0, VA);
            if (z1111) {
                sph(2, k0, VB);
                sph(3, k0, VBB);
                for (int i = 0; i < 3; ++i) {
                    if (ik == 1) {
                        if (i == 0) {
                            Vl[i] = o_lin3(xAA, VAA[i] * sq(r3), xA, VA[i] * sq(r1), xB, VB[i] * sq(r2)) / sq(rr);
                            Vr[i] = o_lin3(xA, VA[i] * sq(r1), xB, VB[i] * sq(r2), xBB, VBB[i] * sq(r4)) / sq(rr);
                        } else {
                            Vl[i] = o_lin3(xAA, VAA[i] * (r3), xA, VA[i] * (r1), xB, VB[i] * (r2)) / (rr);
                            Vr[i] = o_lin3(xA, VA[i] * (r1), xB, VB[i] * (r2), xBB, VBB[i] * (r4)) / (rr);
                        }
                    } else {
                        Vl[i] = o_lin3(xAA, VAA[i], xA, VA[i], xB, VB[i]);
                        Vr[i] = o_lin3(xA, VA[i], xB, VB[i], xBB, VBB[i]);
                    }
                }
                cart(Vl, L, k0);
                cart(Vr, R, k0);
            } else if (z1112) {
                sph(2, k0, VB);
                for (int i = 0; i < 3; ++i) {
                    Vl[i] = o_lin3(xAA, VAA[i], xA, VA[i], xB, VB[i]);
                    Vr[i] = o_lin2(xA, VA[i], xB, VB[i]);
                }
                cart(Vl, L, k0);
                cart(Vr, R, k0);
            } else {  // z1122: left side only; the right side is set per name below
                for (int i = 0; i < 3; ++i) Vl[i] = o_lin2(xAA, VAA[i], xA, VA[i]);
                cart(Vl, L, k0);
            }
        }
        const double g2 = 2.0 * gamma;
        // rho, Q, rho_He scale as r^2 and p as r^(2 gamma) on the all-Zone_1
        // branch; on the Zone_1/Zone_2 branches the r^2 scaling is overwritten
        // by the plain line (the reference's `if` / `if ... else` sequence,
        // Setka_gran_snos.cpp:502-532 and :617-644), so only p is scaled there.
        const int scal[4] = {0, 8, 9, 4};
        for (int q = 0; q < 4; ++q) {
            const int k = scal[q];
            const bool r2g = k == 4;
            if (z1111) {
                if (r2g) {
                    L[k] = o_lin3(xAA, S(k, 0) * std::pow(r3, g2), xA, S(k, 1) * std::pow(r1, g2), xB,
                                  S(k, 2) * std::pow(r2, g2)) / std::pow(rr, g2);
                    R[k] = o_lin3(xA, S(k, 1) * std::pow(r1, g2), xB, S(k, 2) * std::pow(r2, g2), xBB,
                                  S(k, 3) * std::pow(r4, g2)) / std::pow(rr, g2);
                } else {
                    L[k] = o_lin3(xAA, S(k, 0) * sq(r3), xA, S(k, 1) * sq(r1), xB, S(k, 2) * sq(r2)) / sq(rr);
                    R[k] = o_lin3(xA, S(k, 1) * sq(r1), xB, S(k, 2) * sq(r2), xBB, S(k, 3) * sq(r4)) / sq(rr);
                }
            } else if (z1112) {
                if (r2g) {
                    L[k] = o_lin3(xAA, S(k, 0) * std::pow(r3, g2), xA, S(k, 1) * std::pow(r1, g2), xB,
                                  S(k, 2) * std::pow(r2, g2)) / std::pow(rr, g2);
                    R[k] = o_lin2(xA, S(k, 1) * std::pow(r1, g2), xB, S(k, 2) * std::pow(r2, g2)) / std::pow(rr, g2);
                } else {
                    L[k] = o_lin3(xAA, S(k, 0), xA, S(k, 1), xB, S(k, 2));
                    R[k] = o_lin2(xA, S(k, 1), xB, S(k, 2));
                }
            } else {  // z1122
                if (r2g)
                    L[k] = o_lin2(xAA, S(k, 0) * std::pow(r3, g2), xA, S(k, 1) * std::pow(r1, g2)) / std::pow(rr, g2);
                else
                    L[k] = o_lin2(xAA, S(k, 0), xA, S(k, 1));
                R[k] = o_lin2(xB, S(k, 2), xBB, S(k, 3));
            }
        }
        if (z1122)
            for (int k = 1; k < 8; ++k)
                if (k != 4) R[k] = o_lin2(xB, S(k, 2), xBB, S(k, 3));
    } else {
        const bool l2 = (a0 == 2 && a1 == 2 && b1 == 3 && b0 == 3) || (a0 == 3 && a1 == 3 && b1 == 4 && b0 == 4);
        const bool l3 = (a0 == 2 && a1 == 2 && b1 == 2 && b0 == 3) || (a0 == 3 && a1 == 3 && b1 == 3 && b0 == 4);
        const bool l4 = z1222 || (a0 == 2 && a1 == 3 && b1 == 3 && b0 == 3) || (a0 == 3 && a1 == 4 && b1 == 4 && b0 == 4);
        for (int k = 0; k < NV; ++k) {
            if (l2) {
                L[k] = o_lin2(xAA, S(k, 0), xA, S(k, 1));
                R[k] = o_lin2(xB, S(k, 2), xBB, S(k, 3));
            } else if (l3) {
                L[k] = o_lin3(xAA, S(k, 0), xA, S(k, 1), xB, S(k, 2));
                R[k] = o_lin2(xA, S(k, 1), xB, S(k, 2));
            } else if (l4) {
                L[k] = o_lin2(xA, S(k, 1), xB, S(k, 2));
                R[k] = o_lin3(xA, S(k, 1), xB, S(k, 2), xBB, S(k, 3));
            } else {
                L[k] = o_lin3(xAA, S(k, 0), xA, S(k, 1), xB, S(k, 2));
                R[k] = o_lin3(xA, S(k, 1), xB, S(k, 2), xBB, S(k, 3));
            }
        }
    }
    // positivity fall-back to the cell value (:710-720)
    const int fl[4] = {0, 8, 9, 4};
    for (int q = 0; q < 4; ++q) {
        const int k = fl[q];
        if (k >= 8 && k - 8 >= npassive) continue;
        if (L[k] < 0.0000001) L[k] = S(k, 1);
        if (R[k] < 0.0000001) R[k] = S(k, 2);
    }
}

// Per-face flux, restating Setka::Culc_Gran_Potok (Setka_physics.cpp:2280-2571)
// for the plasma: reconstruction, solver choice, chlld, local dt, flux*area,
// Powell PdivB. Writes 11 values per face: rho, Vx, Vy, Vz, p(energy), Bx,
// By, Bz, divB, Q, rho_He (all times area); returns the dt candidate.
static double o_face(const OMesh* M, const OParams* P, const double* st, const double* cc, const double* fc,
                     const double* fn, const double* fa, const double* xyz1, const double* xyz2,
                     int64_t f, double time, double* out, int* err) {
    const int64_t nc = M->ncell;
    const double area = fa[f];
    const double* n = fn + 3 * f;
    double w = 0.0;
    if (P->move) {  // Gran::culc_velosity, Gran.cpp:571-589
        double ddot = 0.0;
        for (int k = 0; k < 4; ++k) {
            const int64_t nd = M->face_nodes[4 * f + k];
            double dx[3];
            for (int j = 0; j < 3; ++j) dx[j] = xyz2[3 * nd + j] - xyz1[3 * nd + j];
            ddot = ddot + (dx[0] * n[0] + dx[1] * n[1] + dx[2] * n[2]);
        }
        w = ddot / 4.0 / time;
    }
    double loc_time = 10000000.0;
    const int type = M->face_type[f];
    const int64_t A = M->face_cells[2 * f];
    const int64_t B = M->face_cells[2 * f + 1];
    double dist = 0.0;
    double L[NV], R[NV];
    if (type == 0) {
        const double dx = cc[3 * A] - cc[3 * B], dy = cc[3 * A + 1] - cc[3 * B + 1], dz = cc[3 * A + 2] - cc[3 * B + 2];
        dist = std::sqrt(dx * dx + dy * dy + dz * dz) / 2.0;
        const int64_t AA = M->face_tvd ? M->face_tvd[2 * f] : -1, BB = M->face_tvd ? M->face_tvd[2 * f + 1] : -1;
        if (P->tvd && M->cell_tvd[A] && M->cell_tvd[B] && (M->face_surf[f] != 2 || P->snos_on_hp) && AA >= 0 &&
            BB >= 0) {
            const int64_t c4[4] = {AA, A, B, BB};
            const int t4[4] = {M->cell_type[AA], M->cell_type[A], M->cell_type[B], M->cell_type[BB]};
            o_snos_tvd(st, nc, c4, t4, cc, fc + 3 * f, P->gamma, P->npassive, L, R);
        } else {
            o_snos_side(st, nc, A, M->cell_type[A], cc, fc + 3 * f, P->gamma, L);
            o_snos_side(st, nc, B, M->cell_type[B], cc, fc + 3 * f, P->gamma, R);
        }
    } else {
        // boundary faces, Setka_gran_snos.cpp:7-65; plasma_condition (Phys_param.cpp:203-206):
        // Inner_Hard 2, Outer_Hard 2, Outer_Soft 1
        for (int k = 0; k < NV; ++k) L[k] = st[k * nc + A];
        if (type == 3) {
            if (P->soft_fixups) {
                if (n[0] < -0.95) {
                    if (L[1] > P->velosity_inf / 7.0) L[1] = P->velosity_inf / 5.0;
                } else {
                    if (L[1] * n[0] + L[2] * n[1] + L[3] * n[2] < 0.0) {
                        L[1] = 0.1 * n[0];
                        L[2] = 0.1 * n[1];
                        L[3] = 0.1 * n[2];
                    }
                }
            }
            for (int k = 0; k < NV; ++k) R[k] = L[k];
        } else {
            const int32_t row = M->face_bc[f];
            if (row < 0) {
                *err = 5;
                return loc_time;
            }
            for (int k = 0; k < NV; ++k) R[k] = M->bc_vals[(int64_t)NV * row + k];
        }
    }
    int method;
    if (P->method_policy == 1) {
        const double bb = ((L[5] * L[5] + L[6] * L[6] + L[7] * L[7]) + (R[5] * R[5] + R[6] * R[6] + R[7] * R[7])) / 2.0;
        const double pp = (L[4] + R[4]) / 2.0;
        method = (bb / kCpi4 / (2.0 * pp) > P->beta_switch) ? 3 : 2;
    } else {
        method = M->face_method[f];
    }
    const int surf = M->face_surf[f];
    const int left_ydar = (surf == 1 && P->TS_hard) ? 1 : 0;
    const int contact = (surf == 2 && P->contact_hard) ? 1 : 0;
    const int nk = P->npassive;
    double q[8], kq[2] = {0.0, 0.0}, ds[3];
    double bn_sum = 0.5 * (n[0] * (L[5] + R[5]) + n[1] * (L[6] + R[6]) + n[2] * (L[7] + R[7]));
    if (surf == 2 && P->bn_in_p_on_hp) {
        // Setka_physics.cpp:2378-2409: magnetic pressure into p, B = 0, the exact
        // gas-dynamic solver; no B or passive flux, PdivB = 0 (:2467-2470)
        double q1[5] = {L[0], L[1], L[2], L[3], L[4]}, q2[5] = {R[0], R[1], R[2], R[3], R[4]};
        q1[4] += (L[5] * L[5] + L[6] * L[6] + L[7] * L[7]) / (8.0 * kPi);
        q2[4] += (R[5] * R[5] + R[6] * R[6] + R[7] * R[7]) / (8.0 * kPi);
        double gd[5], gds[3];
        const int rcg = o_godunov(n, w, q1, q2, P->contact_hard, P->gamma, gd, gds);
        if (rcg) *err = 14 + rcg;
        for (int k = 0; k < 5; ++k) q[k] = gd[k];
        q[5] = q[6] = q[7] = 0.0;
        ds[0] = gds[0];
        ds[1] = gds[1];
        ds[2] = gds[2];
        bn_sum = 0.0;
    } else if (g_ref_riemann) {
        // the reference's own solver (CPU-baseline timing; it exits on errors)
        g_ref_riemann(method, n, w, L, R, 0, 0, nk, L + 8, R + 8, q, kq, ds, left_ydar, contact);
    } else {
        const int rc = o_chlld(method, n, w, L, R, 0, 0, nk, L + 8, R + 8, q, kq, ds, left_ydar, contact, P->gamma);
        if (rc) *err = 10 + rc;
    }
    if (type == 0 && !(M->face_nodt && M->face_nodt[f])) {
        const double dnt = P->KFL * dist / (mx(std::fabs(ds[0]), std::fabs(ds[2])) + std::fabs(w));
        if (dnt < loc_time) loc_time = mn(loc_time, dnt);
    }
    for (int k = 0; k < 8; ++k) out[k] = q[k] * area;
    out[8] = bn_sum * area;
    out[9] = kq[0] * area;
    out[10] = kq[1] * area;
    return loc_time;
}

// Bera multi-fluid charge-exchange sources for the plasma, restating
// Setka::Calc_sourse_MF_Bera (Setka_physics.cpp:766-1258) without pickup ions,
// with U_bera / Um_bera / UE_bera (:746-762), determ_zone (:1427-1482) and
// Phys_param::Plasma_components_1 (Phys_param.cpp:628-665). Returns m_x, m_y,
// m_z, E scaled by n_H_LISM / Kn.
static void o_bera(const OParams* P, const double* prim /*NV*/, int ctype, const double* H /*5*nh*/, double* S) {
    const double rho = prim[0], p = prim[4], Q = prim[8], rho_He = prim[9];
    int zone;
    if (Q / rho < 50.0)
        zone = (ctype == 1) ? 1 : 2;
    else
        zone = (ctype == 4) ? 4 : 3;
    const int zone_ = zone - 1;  // Calc_sourse_MF_Bera passes zone - 1
    const int al = (zone_ <= 2) ? 2 : 1;
    double rho_p = -(kMeDmp * al * rho_He + 4.0 * (-rho + rho_He)) / (4.0 * (1.0 + kMeDmp));
    double T_p = 8.0 * (1.0 + kMeDmp) * p / (8.0 * rho - (7.0 - al + (-1.0 + al) * kMeDmp) * rho_He);
    if (rho_p <= 1e-8) rho_p = 1e-8;
    if (T_p <= 1e-8) T_p = 1e-8;
    if (T_p > 1e5) T_p = 1e5;
    const double Vp[3] = {prim[1], prim[2], prim[3]};
    double mxs = 0.0, mys = 0.0, mzs = 0.0, Es = 0.0;
    for (int h = 0; h < P->nh; ++h) {
        const double rho_h = H[5 * h + 0];
        const double Vh[3] = {H[5 * h + 1], H[5 * h + 2], H[5 * h + 3]};
        const double T_h = 2.0 * H[5 * h + 4] / mx(rho_h, 1e-9);
        const double d[3] = {Vp[0] - Vh[0], Vp[1] - Vh[1], Vp[2] - Vh[2]};
        const double uu = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        // (V2 - V1) has the same norm bitwise, so U is symmetric
        const double U_ph = std::sqrt((4.0 / kPi) * (T_p + T_h) + sq(uu));
        const double U_hp = std::sqrt((4.0 / kPi) * (T_h + T_p) + sq(uu));
        const double Um_ph = std::sqrt((16.0 / kPi) * T_p + (9.0 * kPi / 4.0) * T_h + 4.0 * sq(uu));
        const double Um_hp = std::sqrt((16.0 / kPi) * T_h + (9.0 * kPi / 4.0) * T_p + 4.0 * sq(uu));
        const double UE_ph = std::sqrt((4.0 / kPi) * T_p + (64.0 / 9.0 / kPi) * T_h + sq(uu));
        const double UE_hp = std::sqrt((4.0 / kPi) * T_h + (64.0 / 9.0 / kPi) * T_p + sq(uu));
        const double sig_ph = sq(1.0 - P->par_a_2 * std::log(U_ph));
        const double sig_hp = sq(1.0 - P->par_a_2 * std::log(U_hp));
        const double k_hp = sig_hp * rho_p * rho_h;
        const double k_ph = sig_ph * rho_p * rho_h;
        double Hm_hp[3], Hm_ph[3];
        for (int j = 0; j < 3; ++j) {
            Hm_hp[j] = k_hp * (U_hp * Vp[j] + T_p / Um_hp * (Vp[j] - Vh[j]));
            Hm_ph[j] = k_ph * (U_ph * Vh[j] - T_h / Um_ph * (Vp[j] - Vh[j]));
        }
        const double vp2 = Vp[0] * Vp[0] + Vp[1] * Vp[1] + Vp[2] * Vp[2];
        const double vh2 = Vh[0] * Vh[0] + Vh[1] * Vh[1] + Vh[2] * Vh[2];
        const double vpd = Vp[0] * d[0] + Vp[1] * d[1] + Vp[2] * d[2];
        const double vhd = Vh[0] * d[0] + Vh[1] * d[1] + Vh[2] * d[2];
        const double HE_hp = k_hp * (0.5 * U_hp * vp2 + T_p / Um_hp * vpd + 3.0 / 4.0 * T_p * UE_hp);
        const double HE_ph = k_ph * (0.5 * U_ph * vh2 - T_h / Um_ph * vhd + 3.0 / 4.0 * T_h * UE_ph);
        mxs += (-Hm_hp[0] + Hm_ph[0]);
        mys += (-Hm_hp[1] + Hm_ph[1]);
        mzs += (-Hm_hp[2] + Hm_ph[2]);
        Es += (-HE_hp + HE_ph);
    }
    const double ddp = (P->par_n_H_LISM / P->par_Kn);
    S[0] = mxs * ddp;
    S[1] = mys * ddp;
    S[2] = mzs * ddp;
    S[3] = Es * ddp;
}

// Conservative update of one cell, restating Setka_physics.cpp:1671-2028
// (plasma): flux gather in the cell's face order with sign by cells[0],
// Powell terms, ALE volume ratio, sources, Zone_2 dissipation, floors.
static void o_cell(const OMesh* M, const OParams* P, const double* st, double* st2, const double* H,
                   const double* S_ext, const double* fl, const double* vol1, const double* vol2, int64_t c,
                   double time, int* err, int64_t* nrf, int64_t* npf) {
    const int64_t nc = M->ncell;
    const double Volume = vol1[c];
    const double Volume2 = vol2[c];
    double PO[11];
    for (int k = 0; k < 11; ++k) PO[k] = 0.0;
    for (int s = 0; s < 6; ++s) {
        const int64_t f = M->cell_faces[6 * c + s];
        const double sign = (M->face_cells[2 * f] != c) ? -1.0 : 1.0;
        for (int k = 0; k < 11; ++k) PO[k] += sign * fl[11 * f + k];
    }
    double prim[NV];
    for (int k = 0; k < NV; ++k) prim[k] = st[k * nc + c];
    double S[4] = {0.0, 0.0, 0.0, 0.0};
    if (S_ext) {
        for (int k = 0; k < 4; ++k) S[k] = S_ext[4 * c + k];
    } else if (P->nh > 0) {
        double Hc[20];
        for (int k = 0; k < 5 * P->nh; ++k) Hc[k] = H[(int64_t)k * nc + c];
        o_bera(P, prim, M->cell_type[c], Hc, S);
    }
    const double g1 = P->gamma - 1.0;
    const double rho = prim[0], vx = prim[1], vy = prim[2], vz = prim[3], p = prim[4];
    const double bx = prim[5], by = prim[6], bz = prim[7], Q = prim[8], rho_He = prim[9];
    const double dsk = vx * bx + vy * by + vz * bz;
    double rho3 = rho * Volume / Volume2 - time * PO[0] / Volume2;
    bool rho_null = false;
    double Q3 = 0.0, rho_He3 = 0.0;
    if (rho3 < 1e-7) {
        rho_null = true;
        rho3 = 0.1;
        Q3 = Q / rho * rho3;
        rho_He3 = 0.0;
        (*nrf)++;
    }
    if (P->npassive) {
        Q3 = Q * Volume / Volume2 - time * PO[9] / Volume2;
        rho_He3 = rho_He * Volume / Volume2 - time * PO[10] / Volume2;
    } else {
        Q3 = 0.0;
        rho_He3 = 0.0;
    }
    if (rho_He3 < 0.0) rho_He3 = 0.0;
    double u3, v3, w3, bx3, by3, bz3, p3;
    if (!rho_null) {
        u3 = (rho * vx * Volume / Volume2 - time * (PO[1] + (bx / kCpi4) * PO[8]) / Volume2 + time * S[0]) / rho3;
        v3 = (rho * vy * Volume / Volume2 - time * (PO[2] + (by / kCpi4) * PO[8]) / Volume2 + time * S[1]) / rho3;
        w3 = (rho * vz * Volume / Volume2 - time * (PO[3] + (bz / kCpi4) * PO[8]) / Volume2 + time * S[2]) / rho3;
        bx3 = bx * Volume / Volume2 - time * (PO[5] + vx * PO[8]) / Volume2;
        by3 = by * Volume / Volume2 - time * (PO[6] + vy * PO[8]) / Volume2;
        bz3 = bz * Volume / Volume2 - time * (PO[7] + vz * PO[8]) / Volume2;
        p3 = (((p / g1 + 0.5 * rho * (vx * vx + vy * vy + vz * vz) + (bx * bx + by * by + bz * bz) / kC8Pi) * Volume /
                   Volume2 -
               time * (PO[4] + (dsk / kCpi4) * PO[8]) / Volume2 + time * S[3]) -
              0.5 * rho3 * (u3 * u3 + v3 * v3 + w3 * w3) - (bx3 * bx3 + by3 * by3 + bz3 * bz3) / kC8Pi) *
             g1;
        if (M->cell_type[c] == 2) {  // Zone_2 effective magnetic dissipation, :1932-1947
            const double tau = 1.0;
            const double bx4 = bx3 - time * bx3 / tau;
            const double by4 = by3 - time * by3 / tau;
            const double bz4 = bz3 - time * bz3 / tau;
            const double p4 =
                p3 + (time / tau - sq(time / tau)) * (g1) * (bx3 * bx3 + by3 * by3 + bz3 * bz3) / (4.0 * kPi);
            bx3 = bx4;
            by3 = by4;
            bz3 = bz4;
            p3 = p4;
        }
    } else {
        u3 = vx;
        v3 = vy;
        w3 = vz;
        bx3 = bx;
        by3 = by;
        bz3 = bz;
        p3 = rho3 / 2.0;
    }
    if (std::isnan(rho3) || std::fpclassify(rho3) == FP_SUBNORMAL || std::isnan(Q3) ||
        std::fpclassify(Q3) == FP_SUBNORMAL)
        *err = 20;
    if (p3 < 0.00000001) {
        p3 = 0.000001;
        (*npf)++;
    }
    if (rho_He3 > rho3) rho_He3 = rho3 * 0.1;
    st2[0 * nc + c] = rho3;
    st2[1 * nc + c] = u3;
    st2[2 * nc + c] = v3;
    st2[3 * nc + c] = w3;
    st2[4 * nc + c] = p3;
    if (M->cell_tvd[c]) {
        st2[5 * nc + c] = bx3;
        st2[6 * nc + c] = by3;
        st2[7 * nc + c] = bz3;
    } else {
        st2[5 * nc + c] = bx;
        st2[6 * nc + c] = by;
        st2[7 * nc + c] = bz;
    }
    st2[8 * nc + c] = Q3;
    st2[9 * nc + c] = rho_He3;
}

// Prescribed radial node motion (the synthetic ALE mesh motion):
// x' = x + dt * amp_i * sin(omega * t + phase_i) * x / |x|.
void oracle_move_nodes(const OMesh* M, const OParams* P, const double* xyz1, double* xyz2, double t,
                       double time) {
    const int64_t nn = M->nnode;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < nn; ++i) {
        const double x = xyz1[3 * i], y = xyz1[3 * i + 1], z = xyz1[3 * i + 2];
        const double amp = M->node_amp ? M->node_amp[i] : 0.0;
        if (amp == 0.0) {
            xyz2[3 * i] = x;
            xyz2[3 * i + 1] = y;
            xyz2[3 * i + 2] = z;
            continue;
        }
        const double r = std::sqrt(x * x + y * y + z * z);
        const double v = amp * std::sin(P->omega * t + M->node_phase[i]);
        const double s = time * v / r;
        xyz2[3 * i] = x + s * x;
        xyz2[3 * i + 1] = y + s * y;
        xyz2[3 * i + 2] = z + s * z;
    }
}

// ---------------------------------------------------------------------------
// Surface-tracking node motion: Setka::Culc_Velocity_surface
// (TITAN/source/Setka_move.cpp:111-1358) and Luch::dvigenie (Luch.cpp:6-739)
// restated for meshes whose rays are straight lines of nodes.
//  * Surface faces (face_surf 1 = TS, 2 = HP, 3 = BS) of a moving surface take
//    the Riemann solver at w = 0 on their reconstructed states (:128-181 TS,
//    :187-361 HP, :363-447 BS) and give each of their four nodes
//    velocity_X * ds * n: ds = dsl on TS, dsc on HP, dsr on BS. HP faces with
//    fewer than four neighbours on the surface are skipped (:192); with
//    null_bn_on_HP the normal B of both cells and of both face states is
//    removed first (:196-224, :279-295); with bn_in_p_on_HP the magnetic
//    pressure goes into p and Godunov_Solver_Alexashov gives dsc (:298-327).
//    A non-finite or subnormal dsc is an error (:329-342; error kind 19).
//    The three surfaces run in the reference's order, so BS sees the HP
//    cells' B as null_bn_on_HP left it.
//  * Each node sums its faces' contributions in ascending face order (the
//    reference sums under a mutex in thread order), divides by their number
//    and moves along its own direction: x' = x + (V . x/|x|) dt x/|x|
//    (:1213-1265); with hp_tail an HP node with x < 0 moves along (0, y, z)
//    instead, the rule of the reference's heliotail, whose rays lie in planes
//    of constant x (:1237-1247).
//    With sglag_TS / sglag_HP a TS / HP node's mean also takes a term toward
//    the sphere fitted through it and its neighbours (centres from
//    oracle_surface_centres); with sglag_BS a BS node with more than five
//    neighbours one toward their mean with its own position.
//  * Along each ray (a shorter one padded with -1) the end nodes and the
//    surface nodes are anchors; every other node keeps its initial fraction
//    of the segment between the anchors around it, on the ray's direction.
//    With M->ray_law the rays follow the reference's A_Luch law instead
//    (o_a_luch_ray).
// ---------------------------------------------------------------------------

// One ray under the A_Luch law of Luch::dvigenie (Luch.cpp:9-152): walks the
// ray's segments in order and places each node the law moves at r * u, from
// the current radii R2, R3, R4 of the ray's TS, HP and BS nodes (their slots
// follow from the node counts). The R1 node and the surface nodes stay.
static void o_a_luch_ray(const double* law, const int32_t* rn, const double* u, double* xyz2) {
    const int M0 = (int)law[0], M1 = (int)law[1], M11 = (int)law[2], M2 = (int)law[3], M3 = (int)law[4],
              M4 = (int)law[5];
    const double R0 = law[6], R1 = law[7], R5 = law[8];
    auto radius = [&](int slot) {
        const double* x = xyz2 + 3 * (int64_t)rn[slot];
        return std::sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
    };
    const double R2 = radius(M0 + M1 + 1), R3 = radius(M0 + M1 + M2 + 2), R4 = radius(M0 + M1 + M2 + M3 + 3);
    auto put = [&](int slot, double r) {
        for (int k = 0; k < 3; ++k) xyz2[3 * (int64_t)rn[slot] + k] = r * u[k];
    };
    for (int j = 0; j < M0; ++j) put(j, R0 + j * (R1 - R0) / M0);
    int num = M0 + 1;
    for (int j = 0; j < M1; ++j) put(num + j, R1 + (j + 1) * (R2 - R1) / (M1 + 1));
    num += M1 + 1;
    const double dr = (R2 - R1) / (M1 + 1);
    for (int j = 0; j < M11; ++j) put(num + j, R2 + dr * (j + 1));
    num += M11;
    {
        const double a = law[9], b = law[10];
        for (int j = 0; j < M2 - M11; ++j) {
            const double s = (j + 1.0) / (M2 - M11 + 1.0);
            const double q1 = 1.0 - 3.0 * s + 2.0 * (s * s), q2 = 1.0 - 2.0 * s;
            const double ss = s * (a * (q1 * q1) +
                                   s * (7.0 + b * (q2 * q2) * (-1.0 + s) - 2.0 * s * (9.0 + 2.0 * s * (-5.0 + 2.0 * s))));
            put(num + j, R2 + dr * M11 + (R3 - R2 - dr * M11) * ss);
        }
    }
    num += (M2 - M11) + 1;
    {
        const double a = law[11], b = law[12];
        for (int j = 0; j < M3; ++j) {
            const double s = (j + 1.0) / (M3 + 1.0);
            const double ss = s * (a - (2.0 * a + b - 3.0) * s + (a + b - 2.0) * s * s);
            put(num + j, R3 + (R4 - R3) * ss);
        }
    }
    num += M3 + 1;
    {
        const double a = law[13], b = 2.0;
        for (int j = 0; j < M4; ++j) {
            const double s = (j + 1.0) / (M4 + 1.0);
            const double ss = a * s - (3.0 * a + b - 4.0) * s * s * s + (2.0 * a + b - 3.0) * s * s * s * s;
            put(num + j, R4 + (R5 - R4) * ss);
        }
    }
    put(num + M4, R5);
}

// Radii and directions of the rays at `xyz` (the start of tracking).
void oracle_ray_geometry(const OMesh* M, const double* xyz, double* r0, double* dir) {
    const int64_t L = M->ray_len;
    for (int64_t r = 0; r < M->nray; ++r) {
        for (int64_t j = 0; j < L; ++j) {
            const int64_t i = M->ray_nodes[r * L + j];
            if (i < 0) {  // padding after a shorter ray's last node
                r0[r * L + j] = 0.0;
                continue;
            }
            const double x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
            r0[r * L + j] = std::sqrt(x * x + y * y + z * z);
        }
        const int64_t i0 = M->ray_nodes[r * L];
        const double x = xyz[3 * i0], y = xyz[3 * i0 + 1], z = xyz[3 * i0 + 2];
        const double n0 = std::sqrt(x * x + y * y + z * z);
        dir[3 * r] = x / n0;
        dir[3 * r + 1] = y / n0;
        dir[3 * r + 2] = z / n0;
    }
}

// A surface node's neighbours for smoothing: the other nodes of its
// surface's faces (Setka::Find_Yzel_Sosed_for_BS, Setka_move.cpp:2365-2397, and
// the same sets in Smooth_head_TS3 / _HP3), ascending node id.
static std::vector<std::vector<int64_t>> o_surface_neighbours_of_nodes(const OMesh* M) {
    const int64_t nn = M->nnode, nf = M->nface;
    std::vector<std::vector<int64_t>> nb(nn);
    for (int64_t f = 0; f < nf; ++f) {
        const int s = M->face_surf[f];
        if (s < 1 || s > 3) continue;
        for (int k = 0; k < 4; ++k)
            for (int j = 0; j < 4; ++j)
                if (j != k) nb[M->face_nodes[4 * f + k]].push_back(M->face_nodes[4 * f + j]);
    }
    for (int64_t i = 0; i < nn; ++i) {
        auto& v = nb[i];
        std::sort(v.begin(), v.end());
        v.erase(std::unique(v.begin(), v.end()), v.end());
        v.erase(std::remove(v.begin(), v.end(), i), v.end());
    }
    return nb;
}

// Weighted least squares of 2 p . c = |p|^2 (normal equations, partial
// pivoting); singular (all weights zero): the zero vector.
static void o_fit_weighted(const std::vector<std::array<double, 3>>& P, const std::vector<double>& w, double c[3]) {
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
        for (int k = 0; k < 3; ++k) scale = mx(scale, std::fabs(M[j][k]));
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

// Sphere centre of Setka::Smooth_head_TS3 / _HP3 (Setka_move.cpp:2205-2362):
// the least-squares c of 2 p . c = |p|^2 over the node and its neighbours, then
// up to 8 fits re-weighted by Tukey's biweight of the distance residuals
// (cutoff 2.5 standard deviations) until the RMS residual changes by less than
// 1e-6 (the reference solves each fit by SVD).
static void o_fit_centre(const std::vector<std::array<double, 3>>& P, double c[3]) {
    const size_t n = P.size();
    std::vector<double> w(n, 1.0), res(n);
    o_fit_weighted(P, w, c);
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
        o_fit_weighted(P, w, c);
    }
}

// Fitted centres of the surface nodes at `xyz` (out: nnode*3, zero elsewhere).
void oracle_surface_centres(const OMesh* M, const double* xyz, double* out) {
    const int64_t nn = M->nnode;
    const auto nb = o_surface_neighbours_of_nodes(M);
    std::fill(out, out + 3 * nn, 0.0);
    for (int64_t i = 0; i < nn; ++i) {
        if (nb[i].empty()) continue;
        std::vector<std::array<double, 3>> P;
        P.push_back({xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]});
        for (int64_t j : nb[i]) P.push_back({xyz[3 * j], xyz[3 * j + 1], xyz[3 * j + 2]});
        o_fit_centre(P, out + 3 * i);
    }
}

// Number of faces of the same surface sharing an edge with each surface face
// (Gran::grans_surf).
static std::vector<int> o_surface_neighbours(const OMesh* M) {
    const int64_t nf = M->nface;
    std::unordered_map<uint64_t, int> edges;
    auto key = [](int64_t a, int64_t b, int s) {
        if (a > b) std::swap(a, b);
        return ((uint64_t)a << 34) ^ ((uint64_t)b << 2) ^ (uint64_t)s;
    };
    for (int64_t f = 0; f < nf; ++f) {
        const int s = M->face_surf[f];
        if (s < 1 || s > 3) continue;
        for (int k = 0; k < 4; ++k) edges[key(M->face_nodes[4 * f + k], M->face_nodes[4 * f + (k + 1) % 4], s)]++;
    }
    std::vector<int> nb(nf, 0);
    for (int64_t f = 0; f < nf; ++f) {
        const int s = M->face_surf[f];
        if (s < 1 || s > 3) continue;
        for (int k = 0; k < 4; ++k)
            nb[f] += edges[key(M->face_nodes[4 * f + k], M->face_nodes[4 * f + (k + 1) % 4], s)] - 1;
    }
    return nb;
}

static bool o_surface_moves(const OParams* P, int s) {
    return (s == 1 && P->move_TS) || (s == 2 && P->move_HP) || (s == 3 && P->move_BS);
}

// Face states of an interior face, as o_face forms them.
static void o_interior_states(const OMesh* M, const OParams* P, const double* st, const double* cc, const double* fc,
                              int64_t f, double* L, double* R) {
    const int64_t nc = M->ncell;
    const int64_t A = M->face_cells[2 * f], B = M->face_cells[2 * f + 1];
    const int64_t AA = M->face_tvd ? M->face_tvd[2 * f] : -1, BB = M->face_tvd ? M->face_tvd[2 * f + 1] : -1;
    if (P->tvd && M->cell_tvd[A] && M->cell_tvd[B] && (M->face_surf[f] != 2 || P->snos_on_hp) && AA >= 0 && BB >= 0) {
        const int64_t c4[4] = {AA, A, B, BB};
        const int t4[4] = {M->cell_type[AA], M->cell_type[A], M->cell_type[B], M->cell_type[BB]};
        o_snos_tvd(st, nc, c4, t4, cc, fc + 3 * f, P->gamma, P->npassive, L, R);
    } else {
        o_snos_side(st, nc, A, M->cell_type[A], cc, fc + 3 * f, P->gamma, L);
        o_snos_side(st, nc, B, M->cell_type[B], cc, fc + 3 * f, P->gamma, R);
    }
}

// One surface-tracking node motion xyz -> xyz2 with the step's dt `time`;
// `st` loses the HP cells' normal B when null_bn_on_HP. Returns an error kind
// (0 ok) and the face in *bad.
static int o_surface_motion(const OMesh* M, const OParams* P, double* st, const double* xyz, double* xyz2,
                            const double* cc, const double* fc, const double* fn, double time, int64_t* bad) {
    const int64_t nn = M->nnode, nf = M->nface, nc = M->ncell;
    const std::vector<int> nb = o_surface_neighbours(M);
    std::vector<int8_t> node_surf(nn, 0);
    std::vector<uint8_t> on(nf, 0);
    for (int64_t f = 0; f < nf; ++f) {
        const int s = M->face_surf[f];
        if (s < 1 || s > 3) continue;
        for (int k = 0; k < 4; ++k) node_surf[M->face_nodes[4 * f + k]] = (int8_t)s;
        if (!o_surface_moves(P, s) || M->face_type[f] != 0) continue;
        if (s == 2 && nb[f] < 4) continue;
        on[f] = 1;
    }
    std::vector<double> vf(3 * nf, 0.0);
    int err = 0;
    for (int s = 1; s <= 3; ++s) {
        const double vel = s == 1 ? P->velocity_TS : (s == 2 ? P->velocity_HP : P->velocity_BS);
#pragma omp parallel for schedule(static)
        for (int64_t f = 0; f < nf; ++f) {
            if (!on[f] || M->face_surf[f] != s) continue;
            const double* n = fn + 3 * f;
            const bool nullbn = (s == 2 && P->null_bn_on_HP);
            if (nullbn) {
                const int64_t cs[2] = {M->face_cells[2 * f], M->face_cells[2 * f + 1]};
                for (int64_t c : cs) {
                    double* bx = st + 5 * nc + c;
                    double* by = st + 6 * nc + c;
                    double* bz = st + 7 * nc + c;
                    const double dtpr = n[0] * *bx + n[1] * *by + n[2] * *bz;
                    *bx -= dtpr * n[0];
                    *by -= dtpr * n[1];
                    *bz -= dtpr * n[2];
                }
            }
            double L[NV], R[NV];
            o_interior_states(M, P, st, cc, fc, f, L, R);
            int method;
            if (P->method_policy == 1) {
                const double bb =
                    ((L[5] * L[5] + L[6] * L[6] + L[7] * L[7]) + (R[5] * R[5] + R[6] * R[6] + R[7] * R[7])) / 2.0;
                const double pp = (L[4] + R[4]) / 2.0;
                method = (bb / kCpi4 / (2.0 * pp) > P->beta_switch) ? 3 : 2;
            } else {
                method = M->face_method[f];
            }
            if (nullbn) {
                for (double* q : {L, R}) {
                    const double dtpr = n[0] * q[5] + n[1] * q[6] + n[2] * q[7];
                    q[5] -= dtpr * n[0];
                    q[6] -= dtpr * n[1];
                    q[7] -= dtpr * n[2];
                }
            }
            double ds[3] = {0.0, 0.0, 0.0}, q[8], kq[2];
            int e = 0;
            if (s == 2 && P->bn_in_p_on_hp) {
                double q1[5] = {L[0], L[1], L[2], L[3], L[4]}, q2[5] = {R[0], R[1], R[2], R[3], R[4]};
                q1[4] += (L[5] * L[5] + L[6] * L[6] + L[7] * L[7]) / (8.0 * kPi);
                q2[4] += (R[5] * R[5] + R[6] * R[6] + R[7] * R[7]) / (8.0 * kPi);
                double gd[5];
                const int rcg = o_godunov(n, 0.0, q1, q2, 0, P->gamma, gd, ds);
                if (rcg) e = 14 + rcg;
            } else {
                const int rc = o_chlld(method, n, 0.0, L, R, 0, 0, 0, nullptr, nullptr, q, kq, ds, 0, 0, P->gamma);
                if (rc) e = 10 + rc;
            }
            if (!e && s == 2 && (std::isnan(ds[1]) || std::fpclassify(ds[1]) == FP_SUBNORMAL)) e = 19;
            const double d = s == 1 ? ds[0] : (s == 2 ? ds[1] : ds[2]);
            for (int k = 0; k < 3; ++k) vf[3 * f + k] = vel * d * n[k];
            if (e) {
#pragma omp critical
                if (!err) {
                    err = e;
                    *bad = f;
                }
            }
        }
    }
    // node velocities: contributions in ascending face order, then the mean
    std::vector<double> V(3 * nn, 0.0);
    std::vector<int> num(nn, 0);
    for (int64_t f = 0; f < nf; ++f) {
        if (!on[f]) continue;
        for (int k = 0; k < 4; ++k) {
            const int64_t i = M->face_nodes[4 * f + k];
            for (int j = 0; j < 3; ++j) V[3 * i + j] += vf[3 * f + j];
            num[i]++;
        }
    }
    std::memcpy(xyz2, xyz, sizeof(double) * 3 * nn);
    const bool smooth = P->sglag_TS || P->sglag_HP || P->sglag_BS;
    const auto nbs = smooth ? o_surface_neighbours_of_nodes(M) : std::vector<std::vector<int64_t>>();
    for (int64_t i = 0; i < nn; ++i) {
        const int s = node_surf[i];
        if (!s || !o_surface_moves(P, s)) continue;
        double v[3] = {V[3 * i], V[3 * i + 1], V[3 * i + 2]};
        int cnt = num[i];
        const double* A = xyz + 3 * i;
        // smoothing (Setka_move.cpp:454-1211): one more term of the mean
        const bool sphere = (s == 1 && P->sglag_TS) || (s == 2 && P->sglag_HP);
        if (sphere && !nbs[i].empty() && M->surf_centre) {
            const double coef = s == 1 ? P->velocity_TS * P->sglag_TS_k_sphere : P->velocity_HP * P->sglag_HP_k_sphere;
            const double* B = M->surf_centre + 3 * i;
            const double rr = std::sqrt((A[0] - B[0]) * (A[0] - B[0]) + (A[1] - B[1]) * (A[1] - B[1]) +
                                        (A[2] - B[2]) * (A[2] - B[2]));
            double r = 0.0;
            for (int64_t j : nbs[i]) {
                const double* X = xyz + 3 * j;
                r += std::sqrt((X[0] - B[0]) * (X[0] - B[0]) + (X[1] - B[1]) * (X[1] - B[1]) +
                               (X[2] - B[2]) * (X[2] - B[2]));
            }
            r /= (int)nbs[i].size();
            const double kk = r / rr;
            for (int k = 0; k < 3; ++k) {
                const double b2 = kk * (A[k] - B[k]) + B[k];
                v[k] += coef * (b2 - A[k]) / time;
            }
            ++cnt;
        } else if (s == 3 && P->sglag_BS && nbs[i].size() > 5) {
            const double coef = P->velocity_BS * P->sglag_BS_k;
            double B[3] = {A[0], A[1], A[2]};
            for (int64_t j : nbs[i])
                for (int k = 0; k < 3; ++k) B[k] += xyz[3 * j + k];
            for (int k = 0; k < 3; ++k) {
                B[k] /= ((int)nbs[i].size() + 1.0);
                v[k] += coef * (B[k] - A[k]) / time;
            }
            ++cnt;
        }
        if (cnt > 0)
            for (double& c : v) c /= cnt;
        // along x / |x|; an HP node of the heliotail (x < 0) along (0, y, z)
        // with hp_tail (Setka_move.cpp:1237-1247), the zero vector (no motion)
        // for a node on the x axis, as Eigen's normalize() leaves it
        double B[3];
        if (P->hp_tail && s == 2 && A[0] < 0.0) {
            const double bn = std::sqrt(A[1] * A[1] + A[2] * A[2]);
            B[0] = 0.0;
            B[1] = bn > 0.0 ? A[1] / bn : 0.0;
            B[2] = bn > 0.0 ? A[2] / bn : 0.0;
        } else {
            const double an = std::sqrt(A[0] * A[0] + A[1] * A[1] + A[2] * A[2]);
            B[0] = A[0] / an;
            B[1] = A[1] / an;
            B[2] = A[2] / an;
        }
        const double vb = v[0] * B[0] + v[1] * B[1] + v[2] * B[2];
        for (int k = 0; k < 3; ++k) xyz2[3 * i + k] = A[k] + vb * time * B[k];
    }
    // rays: the nodes between anchors keep their fraction of the segment
    const int64_t RL = M->ray_len;
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < M->nray; ++r) {
        const int32_t* rn = M->ray_nodes + r * RL;
        const double* r0 = M->ray_r0 + r * RL;
        const double* u = M->ray_dir + 3 * r;
        if (M->ray_law) {
            o_a_luch_ray(M->ray_law, rn, u, xyz2);
            continue;
        }
        int64_t Lr = 0;
        while (Lr < RL && rn[Lr] >= 0) ++Lr;
        int64_t a = 0;
        for (int64_t b = 1; b < Lr; ++b) {
            if (b != Lr - 1 && !node_surf[rn[b]]) continue;
            const double* xa = xyz2 + 3 * (int64_t)rn[a];
            const double* xb = xyz2 + 3 * (int64_t)rn[b];
            const double ra = std::sqrt(xa[0] * xa[0] + xa[1] * xa[1] + xa[2] * xa[2]);
            const double rb = std::sqrt(xb[0] * xb[0] + xb[1] * xb[1] + xb[2] * xb[2]);
            for (int64_t j = a + 1; j < b; ++j) {
                const double rj = ra + (r0[j] - r0[a]) / (r0[b] - r0[a]) * (rb - ra);
                for (int k = 0; k < 3; ++k) xyz2[3 * (int64_t)rn[j] + k] = rj * u[k];
            }
            a = b;
        }
    }
    return err;
}

// Second-order neighbours of every face, restating Setka::Init_TVD
// (Setka_physics.cpp:646-738) on the geometry of `xyz`: beyond each side,
// the neighbour through another face of that cell whose centre direction
// from the face centre is most opposite to the side's outward normal (the
// first minimum in the cell's face order), dropped when that direction is
// within acos(0.1) of the face plane. out: nface*2 (AA, BB), -1 when absent.
void oracle_tvd_neighbours(const OMesh* M, const double* xyz, int32_t* out) {
    const int64_t nc = M->ncell, nf = M->nface;
    std::vector<double> cc(3 * nc), vol(nc), fc(3 * nf), fn(3 * nf), fa(nf);
    oracle_geometry(M, xyz, cc.data(), vol.data(), fc.data(), fn.data(), fa.data());
    auto normalized = [](double* v) {
        const double z = (v[0] * v[0] + v[1] * v[1]) + v[2] * v[2];
        if (z > 0.0) {
            const double s = std::sqrt(z);
            v[0] = v[0] / s;
            v[1] = v[1] / s;
            v[2] = v[2] / s;
        }
    };
    auto dot = [](const double* a, const double* b) { return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]; };
#pragma omp parallel for schedule(static)
    for (int64_t f = 0; f < nf; ++f) {
        const double* G = fc.data() + 3 * f;
        double nrm[3] = {fn[3 * f], fn[3 * f + 1], fn[3 * f + 2]};
        out[2 * f] = out[2 * f + 1] = -1;
        for (int side = 0; side < 2; ++side) {
            const int64_t A = M->face_cells[2 * f + side];
            if (A < 0) break;
            double vec[3] = {nrm[0], nrm[1], nrm[2]};
            if (side == 1)
                for (int j = 0; j < 3; ++j) vec[j] = vec[j] * -1.0;
            double best = 2.0;
            int64_t pick = -1;
            for (int k = 0; k < 6; ++k) {
                const int64_t g = M->cell_faces[6 * A + k];
                if (g == f) continue;
                const int64_t g0 = M->face_cells[2 * g], g1 = M->face_cells[2 * g + 1];
                if (g1 < 0) continue;  // boundary face: no neighbour (Get_Sosed)
                const int64_t cel = g0 == A ? g1 : g0;
                double u[3] = {cc[3 * cel] - G[0], cc[3 * cel + 1] - G[1], cc[3 * cel + 2] - G[2]};
                normalized(u);
                const double cosine = dot(vec, u);
                if (cosine < best) {
                    best = cosine;
                    pick = cel;
                }
            }
            out[2 * f + side] = (int32_t)pick;
        }
        if (M->face_cells[2 * f + 1] < 0) continue;
        // direction checks against the face normal (:724-736)
        for (int side = 0; side < 2; ++side) {
            const int64_t cel = out[2 * f + side];
            if (cel < 0) continue;
            double k3[3] = {cc[3 * cel] - G[0], cc[3 * cel + 1] - G[1], cc[3 * cel + 2] - G[2]};
            normalized(k3);
            const double d = dot(nrm, k3);
            if ((side == 0 ? -d : d) < 0.1) out[2 * f + side] = -1;
        }
    }
}

// Reconstructed face states of every interior face at layer `xyz` (the
// states Culc_Gran_Potok hands to the Riemann solver): LR [nface][2][NV];
// boundary faces are left untouched. used [nface]: 1 where the second-order
// branch ran.
void oracle_face_states(const OMesh* M, const OParams* P, const double* st, const double* xyz, double* LR,
                        int8_t* used) {
    const int64_t nc = M->ncell, nf = M->nface;
    std::vector<double> cc(3 * nc), vol(nc), fc(3 * nf), fn(3 * nf), fa(nf);
    oracle_geometry(M, xyz, cc.data(), vol.data(), fc.data(), fn.data(), fa.data());
#pragma omp parallel for schedule(static)
    for (int64_t f = 0; f < nf; ++f) {
        used[f] = 0;
        if (M->face_type[f] != 0) continue;
        const int64_t A = M->face_cells[2 * f], B = M->face_cells[2 * f + 1];
        double* L = LR + 2 * NV * f;
        double* R = L + NV;
        const int64_t AA = M->face_tvd ? M->face_tvd[2 * f] : -1, BB = M->face_tvd ? M->face_tvd[2 * f + 1] : -1;
        if (P->tvd && M->cell_tvd[A] && M->cell_tvd[B] && (M->face_surf[f] != 2 || P->snos_on_hp) && AA >= 0 &&
            BB >= 0) {
            const int64_t c4[4] = {AA, A, B, BB};
            const int t4[4] = {M->cell_type[AA], M->cell_type[A], M->cell_type[B], M->cell_type[BB]};
            o_snos_tvd(st, nc, c4, t4, cc.data(), fc.data() + 3 * f, P->gamma, P->npassive, L, R);
            used[f] = 1;
        } else {
            o_snos_side(st, nc, A, M->cell_type[A], cc.data(), fc.data() + 3 * f, P->gamma, L);
            o_snos_side(st, nc, B, M->cell_type[B], cc.data(), fc.data() + 3 * f, P->gamma, R);
        }
    }
}

// Flux of every face at layer `xyz1` (and node displacement to `xyz2` when
// moving). fl: 11*nface. Returns the dt candidate (min over Us faces).
double oracle_face_fluxes(const OMesh* M, const OParams* P, const double* st, const double* xyz1,
                          const double* xyz2, double time, double* fl, int* err_out) {
    const int64_t nc = M->ncell, nf = M->nface;
    std::vector<double> cc(3 * nc), vol(nc), fc(3 * nf), fn(3 * nf), fa(nf);
    oracle_geometry(M, xyz1, cc.data(), vol.data(), fc.data(), fn.data(), fa.data());
    double loc = 100000000.0;
    int err = 0;
#pragma omp parallel for schedule(static) reduction(min : loc)
    for (int64_t f = 0; f < nf; ++f) {
        int e = 0;
        const double d = o_face(M, P, st, cc.data(), fc.data(), fn.data(), fa.data(), xyz1, xyz2, f, time,
                                fl + 11 * f, &e);
        if (d < loc) loc = d;
        if (e) {
#pragma omp critical
            if (!err) err = e;
        }
    }
    *err_out = err;
    return loc;
}

// Bera sources for every cell (m_x, m_y, m_z, E): S[4*ncell].
void oracle_sources(const OMesh* M, const OParams* P, const double* st, const double* H, double* S) {
    const int64_t nc = M->ncell;
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < nc; ++c) {
        double prim[NV], Hc[20];
        for (int k = 0; k < NV; ++k) prim[k] = st[k * nc + c];
        for (int k = 0; k < 5 * P->nh; ++k) Hc[k] = H[(int64_t)k * nc + c];
        o_bera(P, prim, M->cell_type[c], Hc, S + 4 * c);
    }
}

// `nsteps` steps of Setka::Go's plasma loop (Setka_physics.cpp:1589-2028).
//   state  [NV*ncell]   in/out (primitive variables)
//   xyz    [3*nnode]    in/out node coordinates (moved when P->move)
//   H      [5*nh*ncell] frozen neutral fluids (may be null when nh == 0)
//   S_ext  [4*ncell]    external sources (overrides Bera when non-null)
//   clock  [2]          in/out: {dt of the next step, physical time t}
// The first step of a run uses the dt the caller passes (the reference starts
// with 1e-5, :1582-1583); each step's CFL minimum is applied on the next step.
int oracle_go(const OMesh* M, const OParams* P, double* state, double* xyz, const double* H, const double* S_ext,
              int64_t nsteps, double* clock, OStepInfo* info) {
    const int64_t nc = M->ncell, nf = M->nface, nn = M->nnode;
    // Scratch kept between calls (every element a step reads is written
    // earlier in the same call), so a call's cost is its steps, not the
    // allocation and first touch of its arrays.
    static thread_local struct {
        std::vector<double> st2, xyz2, fl, cc1, vol1, fc1, fn1, fa1, cc2, vol2, fc2, fn2, fa2;
    } W;
    auto sized = [](std::vector<double>& v, int64_t n) -> std::vector<double>& {
        if ((int64_t)v.size() != n) v.resize(n);
        return v;
    };
    std::vector<double>&st2 = sized(W.st2, NV * nc), &xyz2 = sized(W.xyz2, 3 * nn), &fl = sized(W.fl, 11 * nf);
    std::vector<double>&cc1 = sized(W.cc1, 3 * nc), &vol1 = sized(W.vol1, nc), &fc1 = sized(W.fc1, 3 * nf),
    &fn1 = sized(W.fn1, 3 * nf), &fa1 = sized(W.fa1, nf);
    std::vector<double>&cc2 = sized(W.cc2, 3 * nc), &vol2 = sized(W.vol2, nc), &fc2 = sized(W.fc2, 3 * nf),
    &fn2 = sized(W.fn2, 3 * nf), &fa2 = sized(W.fa2, nf);
    double time = clock[0], tphys = clock[1];
    info->err_code = 0;
    info->n_rho_floor = 0;
    info->n_p_floor = 0;
    oracle_geometry(M, xyz, cc1.data(), vol1.data(), fc1.data(), fn1.data(), fa1.data());
    for (int64_t step = 0; step < nsteps; ++step) {
        const double* X2 = xyz;
        const double* V2 = vol1.data();
        int err = 0;
        if (P->move) {
            if (P->surface_motion) {
                int64_t bad = -1;
                err = o_surface_motion(M, P, state, xyz, xyz2.data(), cc1.data(), fc1.data(), fn1.data(), time, &bad);
                if (err) info->err_index = bad;
            } else {
                oracle_move_nodes(M, P, xyz, xyz2.data(), tphys, time);
            }
            oracle_geometry(M, xyz2.data(), cc2.data(), vol2.data(), fc2.data(), fn2.data(), fa2.data());
            X2 = xyz2.data();
            V2 = vol2.data();
        }
        double loc = 100000000.0;
#pragma omp parallel for schedule(static) reduction(min : loc)
        for (int64_t f = 0; f < nf; ++f) {
            int e = 0;
            const double d = o_face(M, P, state, cc1.data(), fc1.data(), fn1.data(), fa1.data(), xyz, X2, f, time,
                                    fl.data() + 11 * f, &e);
            if (d < loc) loc = d;
            if (e) {
#pragma omp critical
                if (!err) {
                    err = e;
                    info->err_index = f;
                }
            }
        }
        int64_t nrf = 0, npf = 0;
#pragma omp parallel for schedule(static) reduction(+ : nrf, npf)
        for (int64_t c = 0; c < nc; ++c) {
            int e = 0;
            o_cell(M, P, state, st2.data(), H, S_ext, fl.data(), vol1.data(), V2, c, time, &e, &nrf, &npf);
            if (e) {
#pragma omp critical
                if (!err) {
                    err = e;
                    info->err_index = c;
                }
            }
        }
        info->n_rho_floor += nrf;
        info->n_p_floor += npf;
        std::memcpy(state, st2.data(), sizeof(double) * NV * nc);
        if (P->move) {
            std::memcpy(xyz, xyz2.data(), sizeof(double) * 3 * nn);
            cc1.swap(cc2);
            vol1.swap(vol2);
            fc1.swap(fc2);
            fn1.swap(fn2);
            fa1.swap(fa2);
        }
        tphys += time;
        time = loc;
        info->steps_done = step + 1;
        if (err) {
            info->err_code = err;
            break;
        }
    }
    clock[0] = time;
    clock[1] = tphys;
    return (int)info->err_code;
}

int oracle_chlld(int n_state, const double* nrm, double w, const double* q1, const double* q2, int null_bn,
                 int n_disc, int nk, const double* kl, const double* kr, double* qout, double* kout, double* ds,
                 int left_ydar, int contact, double gamma) {
    return o_chlld(n_state, nrm, w, q1, q2, null_bn, n_disc, nk, kl, kr, qout, kout, ds, left_ydar, contact,
                   gamma);
}

void oracle_chlld_batch(int64_t n, const int* n_state, const double* nrm, const double* w, const double* q1,
                        const double* q2, double* qout, double* ds, double gamma, int* rc) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        double dummy = 0.0;
        rc[i] = o_chlld(n_state[i], nrm + 3 * i, w[i], q1 + 8 * i, q2 + 8 * i, 0, 0, 0, &dummy, &dummy,
                        qout + 8 * i, &dummy, ds + 3 * i, 0, 0, gamma);
    }
}

int oracle_godunov(const double* nrm, double w, const double* q1, const double* q2, int contact, double gamma,
                   double* out, double* ds) {
    return o_godunov(nrm, w, q1, q2, contact, gamma, out, ds);
}

void oracle_set_reference_riemann(void* fn) { g_ref_riemann = reinterpret_cast<RefRiemann>(fn); }

int oracle_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// ---------------------------------------------------------------------------
// Monte-Carlo neutral hydrogen pass (the closure's source generator), a CPU
// restatement of the device pass of titan_mc_sources on the same numbering:
//  * the neutral physics of Setka::MK_fly_immit (TITAN/source/Setka_MK.cpp:
//    1752-2314): straight flight through the cells, the charge-exchange rate
//    nu = rho_Th uz sigma(uz) / Kn with uz = Velosity_1(|v - V_p|, cp)
//    (Setka_MK.cpp:40-50, 1976-1988), sigma(u) = (1 - a2 ln u)^2
//    (Phys_param.h:177-180), the optical depth against -ln(1 - xi), the new
//    velocity by the rejection scheme of Setka::M_K_Change_Velosity
//    (Setka_MK.cpp:2788-2852), rho_Th / p_Th of Phys_param::Plasma_components_1
//    (Phys_param.cpp:628-665) with the cell type as zone (Setka_MK.cpp:1956),
//    floored as at Setka_MK.cpp:1966-1967;
//  * the momentum and energy tallies mu (v_old - v_new), mu (|v_old|^2 -
//    |v_new|^2) / 2 per exchange, and mu t per cell (n_H), divided by the
//    cell volume at the end;
//  * inflow: a drifting Maxwellian through the faces whose type is selected,
//    faces chosen by the inflow CDF (stratified by particle id), positions
//    uniform on the quad, velocities flux-weighted by rejection;
//  * random numbers: the counter-based SplitMix64 finaliser over (seed,
//    particle id, draw counter), so every neutral's history is a function of
//    its id alone, and the CDF summed in the same fixed tree as the device
//    scan (warp shuffles of 32, warp totals in order, 256-face rounds of
//    4096-face blocks, blocks combined by 1024 segments).
// The device tracer is compiled with FMA contraction and CUDA's libm, this
// one without contraction and with glibc: a neutral's history agrees to
// rounding until a decision (exchange or not, which face it leaves by, a
// rejection test) falls within rounding of its threshold, so the test
// compares neutrals one by one and requires nearly all to agree.
// ---------------------------------------------------------------------------
namespace {

const double kMcSqrtPi = 1.77245385;                 // sqrtpi_ of TITAN/source/Header.h:94
const double kMcSqrtPiFull = 1.7724538509055160273;  // sqrt(pi) of the inflow flux

struct OMcRng {
    uint64_t key, ctr;
    double uniform() {
        uint64_t z = key + 0x9E3779B97F4A7C15ull * (++ctr);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z = z ^ (z >> 31);
        return ((double)(z >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    }
};

double o_velosity_1(double u, double cp) {
    if (u < 0.00001)
        return 2.0 * cp / kMcSqrtPi + 2.0 * u * u / (3.0 * cp * kMcSqrtPi) - u * u * u * u / (15.0 * cp * cp * cp * kMcSqrtPi);
    return std::exp(-u * u / (cp * cp)) * cp / kMcSqrtPi + (u + (cp * cp) / (2.0 * u)) * std::erf(u / cp);
}

double o_mc_sigma(double a2, double x) {
    const double s = 1.0 - a2 * std::log(x);
    return s * s;
}

void o_change_velocity(OMcRng& rng, double a2, double cp, const double U[3], const double Vn[3], double W[3]) {
    const double X = std::sqrt((Vn[0] - U[0]) * (Vn[0] - U[0]) + (Vn[1] - U[1]) * (Vn[1] - U[1]) +
                               (Vn[2] - U[2]) * (Vn[2] - U[2]));
    const double p4 = 0.5 * kMcSqrtPi * X / (1.0 + 0.5 * kMcSqrtPi * X);
    double v1 = U[0], v2 = U[1], v3 = U[2];
    for (int it = 0; it < 1000; ++it) {
        const double k1 = rng.uniform(), k2 = rng.uniform(), k3 = rng.uniform();
        const double k4 = rng.uniform(), k5 = rng.uniform(), k6 = rng.uniform();
        double y1, y2, y3;
        if (p4 < k1) {
            const double om1 = 1.0 - 2.0 * k4;
            const double so = std::sqrt(1.0 - om1 * om1);
            const double om2 = so * std::cos(2.0 * kPi * k5), om3 = so * std::sin(2.0 * kPi * k5);
            const double lo = std::sqrt(-std::log(k2 * k3));
            y1 = lo * om1;
            y2 = lo * om2;
            y3 = lo * om3;
        } else {
            y1 = std::sqrt(-std::log(k2)) * std::cos(kPi * k3);
            y2 = std::sqrt(-std::log(k4)) * std::cos(2.0 * kPi * k5);
            y3 = std::sqrt(-std::log(k4)) * std::sin(2.0 * kPi * k5);
        }
        v1 = y1 + U[0];
        v2 = y2 + U[1];
        v3 = y3 + U[2];
        const double u1 = Vn[0] - v1, u2 = Vn[1] - v2, u3 = Vn[2] - v3;
        const double uuu = std::sqrt(u1 * u1 + u2 * u2 + u3 * u3);
        const double yy = std::sqrt(y1 * y1 + y2 * y2 + y3 * y3);
        const double h = (uuu * o_mc_sigma(a2, uuu * cp)) / (o_mc_sigma(a2, X * cp) * (X + yy));
        if (!(h < k6)) break;
    }
    W[0] = v1;
    W[1] = v2;
    W[2] = v3;
}

// The device's block scan of NT values v[0..NT): inclusive scan within each
// warp of 32 (shuffle steps 1, 2, 4, 8, 16), then each warp adds the totals of
// the warps before it, summed in ascending order. Returns the block total.
double o_block_scan(std::vector<double>& v) {
    const size_t nt = v.size(), nw = nt / 32;
    std::vector<double> prev(nt), wt(nw);
    for (int o = 1; o < 32; o <<= 1) {
        prev = v;
        for (size_t t = 0; t < nt; ++t)
            if ((int)(t & 31) >= o) v[t] = prev[t] + prev[t - o];
    }
    for (size_t w = 0; w < nw; ++w) wt[w] = v[32 * w + 31];
    double all = 0.0;
    for (size_t k = 0; k < nw; ++k) all += wt[k];
    for (size_t t = 0; t < nt; ++t) {
        double before = 0.0;
        for (size_t k = 0; k < t / 32; ++k) before += wt[k];
        v[t] = before + v[t];
    }
    return all;
}

}  // namespace

// One pass over a stationary mesh (its geometry formed here as
// oracle_geometry does). tally [5][ncell] (n_H, S_m (3), S_E per unit volume),
// trace [nparticles][8] or null (the device's per-neutral end record),
// *inflow_total the neutrals entering per unit time, *lost the neutrals that
// ended other than through the boundary. Returns 0, or 1 when no face lets
// neutrals in.
// Tabulated inflow of some faces (the reference's face AMR functions as
// input, Setka_MK.cpp:1225-1575): per face its frame Vn, Vt, Vm, the side the
// neutrals enter and its leaves (box in local velocities, value f) in tree order.
struct OMcFaceDist {
    int64_t nface;
    const int32_t* face;
    const int8_t* side;
    const double* frame;
    const int64_t* leaf_ptr;
    const double* leaf_box;
    const double* leaf_f;
};

// Outgoing tallies on some faces (AMR_f::Add_particle, AMR_f.cpp:240-316, at
// Setka_MK.cpp:2165-2182): per face the side whose leaving neutrals stop
// there, the frame and the leaf boxes. Results: leaf weights, moments (n,
// Smu, nn) per face, and the neutrals no leaf held.
struct OMcFaceTally {
    int64_t nface;
    const int32_t* face;
    const int8_t* side;
    const double* frame;
    const int64_t* leaf_ptr;
    const double* leaf_box;
    double* leaf_f;
    double* moments;
    int64_t* unplaced;
};

int oracle_mc_pass(const OMesh* M, const double* xyz, const double* state, int32_t npassive, double par_a_2,
                   double par_Kn, double nH, const double* uH, double cpH, uint32_t face_types, uint64_t seed,
                   int64_t nparticles, int32_t max_cells, double* tally, double* trace, double* inflow_total,
                   int64_t* lost_out, const OMcFaceDist* fd, const OMcFaceTally* ft) {
    const int64_t nc = M->ncell, nf = M->nface;
    std::vector<double> cc(3 * nc), vol(nc), fc(3 * nf), fn(3 * nf), fa(nf);
    oracle_geometry(M, xyz, cc.data(), vol.data(), fc.data(), fn.data(), fa.data());
    // the tables: each leaf's weight box volume * f * |centre x| (Culk_SpotokV,
    // AMR_f.cpp:4-48), the face's inflow per unit area and the leaves'
    // cumulative shares (the last one 1)
    std::vector<int64_t> tab_of(nf, -1);
    std::vector<double> tab_flux, leaf_cum;
    if (fd && fd->nface > 0) {
        tab_flux.resize(fd->nface);
        leaf_cum.resize(fd->leaf_ptr[fd->nface]);
        for (int64_t i = 0; i < fd->nface; ++i) {
            tab_of[fd->face[i]] = i;
            double sum = 0.0;
            for (int64_t l = fd->leaf_ptr[i]; l < fd->leaf_ptr[i + 1]; ++l) {
                const double* b = fd->leaf_box + 6 * l;
                const double dx = b[1] - b[0], dy = b[3] - b[2], dz = b[5] - b[4];
                sum += dx * dy * dz * fd->leaf_f[l] * std::fabs((b[0] + b[1]) / 2.0);
                leaf_cum[l] = sum;
            }
            tab_flux[i] = sum;
            for (int64_t l = fd->leaf_ptr[i]; l < fd->leaf_ptr[i + 1]; ++l)
                leaf_cum[l] = (l == fd->leaf_ptr[i + 1] - 1) ? 1.0 : leaf_cum[l] / sum;
        }
    }
    // inflow weights and their CDF, in the device's summation tree
    auto weight = [&](int64_t f) {
        if (tab_of[f] >= 0) return tab_flux[tab_of[f]] * fa[f];
        const int t = M->face_type[f];
        if (t <= 0 || t > 31 || !((face_types >> t) & 1u)) return 0.0;
        const double un = -(uH[0] * fn[3 * f] + uH[1] * fn[3 * f + 1] + uH[2] * fn[3 * f + 2]);
        const double sr = un / cpH;
        const double flux = nH * (cpH * std::exp(-sr * sr) / (2.0 * kMcSqrtPiFull) + 0.5 * un * (1.0 + std::erf(sr)));
        return flux * fa[f];
    };
    const int64_t kChunk = 4096, kRound = 256, kSeg = 1024;
    const int64_t nb = (nf + kChunk - 1) / kChunk;
    std::vector<double> cdf(nf), bs(nb);
    std::vector<double> v(kRound);
    for (int64_t b = 0; b < nb; ++b) {
        double carry = 0.0;
        for (int64_t r = 0; r < kChunk / kRound; ++r) {
            for (int64_t t = 0; t < kRound; ++t) {
                const int64_t f = b * kChunk + r * kRound + t;
                v[t] = f < nf ? weight(f) : 0.0;
            }
            const double all = o_block_scan(v);
            for (int64_t t = 0; t < kRound; ++t) {
                const int64_t f = b * kChunk + r * kRound + t;
                if (f < nf) cdf[f] = carry + v[t];
            }
            carry += all;
        }
        bs[b] = carry;
    }
    const int64_t per = (nb + kSeg - 1) / kSeg;
    std::vector<double> seg(kSeg), incl(kSeg);
    for (int64_t t = 0; t < kSeg; ++t) {
        const int64_t b0 = std::min(nb, t * per), b1 = std::min(nb, b0 + per);
        double sg = 0.0;
        for (int64_t b = b0; b < b1; ++b) {
            const double x = bs[b];
            bs[b] = sg;
            sg += x;
        }
        seg[t] = sg;
    }
    incl = seg;
    const double total = o_block_scan(incl);
    for (int64_t t = 0; t < kSeg; ++t) {
        const int64_t b0 = std::min(nb, t * per), b1 = std::min(nb, b0 + per);
        const double before = incl[t] - seg[t];
        for (int64_t b = b0; b < b1; ++b) bs[b] += before;
    }
    if (!(total > 0.0)) return 1;
    for (int64_t f = 0; f < nf; ++f) cdf[f] = (f == nf - 1) ? 1.0 : (cdf[f] + bs[f / kChunk]) / total;
    *inflow_total = total;
    const double mu = total / (double)nparticles;
    // the tracing records: outward face planes, neighbours, proton fluid
    std::vector<double> plane(24 * nc), fluid(5 * nc);
    std::vector<int32_t> nbr(6 * nc);
    for (int64_t c = 0; c < nc; ++c) {
        for (int sl = 0; sl < 6; ++sl) {
            const int64_t f = M->cell_faces[6 * c + sl];
            const bool first = M->face_cells[2 * f] == c;
            const double sg = first ? 1.0 : -1.0;
            const double n0 = sg * fn[3 * f], n1 = sg * fn[3 * f + 1], n2 = sg * fn[3 * f + 2];
            double* P = &plane[24 * c + 4 * sl];
            P[0] = n0;
            P[1] = n1;
            P[2] = n2;
            P[3] = fc[3 * f] * n0 + fc[3 * f + 1] * n1 + fc[3 * f + 2] * n2;
            nbr[6 * c + sl] = first ? M->face_cells[2 * f + 1] : M->face_cells[2 * f];
            if (ft)  // a tallied face seen from its side cell: neutrals stop there (table t as -3 - t)
                for (int64_t t = 0; t < ft->nface; ++t)
                    if (ft->face[t] == f && ft->side[t] == (first ? 0 : 1)) nbr[6 * c + sl] = (int32_t)(-3 - t);
        }
        const double rho = state[c], p = state[4 * nc + c];
        const double rho_He = npassive ? state[9 * nc + c] : 0.0;
        const int al = (M->cell_type[c] <= 2) ? 2 : 1;
        double r = -(kMeDmp * al * rho_He + 4.0 * (-rho + rho_He)) / (4.0 * (1.0 + kMeDmp));
        double pt = p * (4.0 * rho - (4.0 + al * kMeDmp) * rho_He) / (8.0 * rho + (-7.0 + al + (1.0 - al) * kMeDmp) * rho_He);
        if (r <= 1e-8) r = 1e-8;
        if (pt <= 1e-8 / 2.0) pt = 1e-8 / 2.0;
        fluid[5 * c] = r;
        fluid[5 * c + 1] = std::sqrt(2.0 * pt / r);
        fluid[5 * c + 2] = state[nc + c];
        fluid[5 * c + 3] = state[2 * nc + c];
        fluid[5 * c + 4] = state[3 * nc + c];
    }
    std::fill(tally, tally + 5 * nc, 0.0);
    int64_t lost = 0;
    // the tallied faces' bounds (the leaves' bounding box) and their accumulators
    std::vector<double> ft_bounds;
    if (ft) {
        ft_bounds.resize(6 * ft->nface);
        for (int64_t t = 0; t < ft->nface; ++t) {
            double* B = &ft_bounds[6 * t];
            for (int k = 0; k < 6; k += 2) {
                B[k] = HUGE_VAL;
                B[k + 1] = -HUGE_VAL;
            }
            for (int64_t l = ft->leaf_ptr[t]; l < ft->leaf_ptr[t + 1]; ++l)
                for (int k = 0; k < 6; k += 2) {
                    B[k] = std::min(B[k], ft->leaf_box[6 * l + k]);
                    B[k + 1] = std::max(B[k + 1], ft->leaf_box[6 * l + k + 1]);
                }
        }
        std::fill(ft->leaf_f, ft->leaf_f + ft->leaf_ptr[ft->nface], 0.0);
        std::fill(ft->moments, ft->moments + 3 * ft->nface, 0.0);
        *ft->unplaced = 0;
    }
    auto stop_on_face = [&](int64_t t, const double* v) {
        const double* E = ft->frame + 9 * t;
        const double Vnn = std::fabs(v[0] * E[0] + v[1] * E[1] + v[2] * E[2]);
        ft->moments[3 * t] += mu / Vnn;
        ft->moments[3 * t + 1] += mu;
        ft->moments[3 * t + 2] += mu * ((1.0 / Vnn) * (1.0 / Vnn));
        double q[3] = {v[0] * E[0] + v[1] * E[1] + v[2] * E[2], v[0] * E[3] + v[1] * E[4] + v[2] * E[5],
                       v[0] * E[6] + v[1] * E[7] + v[2] * E[8]};
        const double* B = &ft_bounds[6 * t];
        for (int k = 0; k < 3; ++k) {
            if (q[k] < B[2 * k]) q[k] = B[2 * k] + 1e-7;
            if (q[k] > B[2 * k + 1]) q[k] = B[2 * k + 1] - 1e-7;
        }
        for (int kk = 1; kk <= 30; ++kk) {
            for (int64_t l = ft->leaf_ptr[t]; l < ft->leaf_ptr[t + 1]; ++l) {
                const double* b = ft->leaf_box + 6 * l;
                if (b[0] <= q[0] && q[0] < b[1] && b[2] <= q[1] && q[1] < b[3] && b[4] <= q[2] && q[2] < b[5]) {
                    ft->leaf_f[l] += mu;
                    return;
                }
            }
            q[0] *= 0.995;
            if (kk < 20) {
                q[1] *= 0.995;
                q[2] *= 0.995;
            }
        }
        ++*ft->unplaced;
    };
    for (int64_t pid = 0; pid < nparticles; ++pid) {
        OMcRng rng{seed ^ (0xD1B54A32D192ED03ull * (uint64_t)(pid + 1)), 0ull};
        const double s = ((double)pid + rng.uniform()) / (double)nparticles;
        int64_t lo = 0, hi = nf - 1;
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if (cdf[mid] < s)
                lo = mid + 1;
            else
                hi = mid;
        }
        const int64_t f0 = lo;
        double P[4][3];
        for (int k = 0; k < 4; ++k)
            for (int d = 0; d < 3; ++d) P[k][d] = xyz[3 * M->face_nodes[4 * f0 + k] + d];
        const double A1 = tri_area(P[0], P[1], P[2]);
        const double A2 = tri_area(P[0], P[3], P[2]);
        const int tb = (rng.uniform() * (A1 + A2) < A1) ? 1 : 3;
        double b1 = rng.uniform(), b2 = rng.uniform();
        if (b1 + b2 > 1.0) {
            b1 = 1.0 - b1;
            b2 = 1.0 - b2;
        }
        double x[3];
        for (int k = 0; k < 3; ++k) x[k] = P[0][k] + b1 * (P[tb][k] - P[0][k]) + b2 * (P[2][k] - P[0][k]);
        const int64_t tab = tab_of[f0];
        double v[3] = {uH[0], uH[1], uH[2]};
        int64_t cell = M->face_cells[2 * f0];
        if (tab >= 0) {
            // AMR_f::Get_random_velosity (AMR_f.cpp:50-96) over the flattened
            // leaves, then AMR_cell::Get_random_velosity_in_cell (AMR_cell.cpp:273-326)
            const double u = rng.uniform();
            int64_t l = fd->leaf_ptr[tab], h = fd->leaf_ptr[tab + 1] - 1;
            while (l < h) {
                const int64_t mid = (l + h) >> 1;
                if (leaf_cum[mid] < u)
                    l = mid + 1;
                else
                    h = mid;
            }
            const double* B = fd->leaf_box + 6 * l;
            const double L = B[0], R = B[1];
            double w[3];
            w[0] = std::sqrt(L * L + rng.uniform() * (R * R - L * L));
            w[1] = B[2] + rng.uniform() * (B[3] - B[2]);
            w[2] = B[4] + rng.uniform() * (B[5] - B[4]);
            const double* E = fd->frame + 9 * tab;
            for (int k = 0; k < 3; ++k) v[k] = w[0] * E[k] + w[1] * E[3 + k] + w[2] * E[6 + k];
            if (fd->side[tab]) cell = M->face_cells[2 * f0 + 1];
        }
        const double nin[3] = {-fn[3 * f0], -fn[3 * f0 + 1], -fn[3 * f0 + 2]};
        const double un = uH[0] * nin[0] + uH[1] * nin[1] + uH[2] * nin[2];
        const double vmax = std::fmax(un, 0.0) + 6.0 * cpH;
        for (int it = 0; it < 4096 && tab < 0; ++it) {
            const double r1 = std::sqrt(-std::log(rng.uniform())), t1 = 2.0 * kPi * rng.uniform();
            const double r2 = std::sqrt(-std::log(rng.uniform())), t2 = 2.0 * kPi * rng.uniform();
            v[0] = uH[0] + cpH * r1 * std::cos(t1);
            v[1] = uH[1] + cpH * r1 * std::sin(t1);
            v[2] = uH[2] + cpH * r2 * std::cos(t2);
            const double vn = v[0] * nin[0] + v[1] * nin[1] + v[2] * nin[2];
            if (vn > 0.0 && rng.uniform() * vmax < vn) break;
        }
        double ksi = -std::log(1.0 - rng.uniform());
        double I = 0.0;
        int nex = 0, visit = 0, kind = 1;
        for (; visit < max_cells; ++visit) {
            const double* R = &plane[24 * cell];
            double t_exit = 1e300;
            int64_t next = -2;
            for (int sl = 0; sl < 6; ++sl) {
                const double vn = v[0] * R[4 * sl] + v[1] * R[4 * sl + 1] + v[2] * R[4 * sl + 2];
                if (vn <= 0.0) continue;
                const double d = R[4 * sl + 3] - (x[0] * R[4 * sl] + x[1] * R[4 * sl + 1] + x[2] * R[4 * sl + 2]);
                const double t = std::fmax(d, 0.0) / vn;
                if (t < t_exit) {
                    t_exit = t;
                    next = nbr[6 * cell + sl];
                }
            }
            if (next == -2) {
                kind = 2;
                break;
            }
            const double* Fl = &fluid[5 * cell];
            const double rho_th = Fl[0], cp = Fl[1];
            const double du0 = v[0] - Fl[2], du1 = v[1] - Fl[3], du2 = v[2] - Fl[4];
            const double u = std::sqrt(du0 * du0 + du1 * du1 + du2 * du2);
            const double uz = o_velosity_1(u, cp);
            const double nu = rho_th * uz * o_mc_sigma(par_a_2, uz) / par_Kn;
            const double dI = nu * t_exit;
            if (I + dI < ksi) {
                tally[cell] += mu * t_exit;
                I += dI;
                for (int k = 0; k < 3; ++k) x[k] += t_exit * v[k];
                if (next < 0) {
                    kind = 0;
                    if (next <= -3) {
                        stop_on_face(-3 - (int64_t)next, v);
                        kind = 3;
                    }
                    break;
                }
                cell = next;
                continue;
            }
            const double t_ex = (ksi - I) / nu;
            tally[cell] += mu * t_ex;
            for (int k = 0; k < 3; ++k) x[k] += t_ex * v[k];
            const double U[3] = {Fl[2] / cp, Fl[3] / cp, Fl[4] / cp};
            const double Vn[3] = {v[0] / cp, v[1] / cp, v[2] / cp};
            double W[3];
            o_change_velocity(rng, par_a_2, cp, U, Vn, W);
            const double w0 = W[0] * cp, w1 = W[1] * cp, w2 = W[2] * cp;
            tally[nc + cell] += mu * (v[0] - w0);
            tally[2 * nc + cell] += mu * (v[1] - w1);
            tally[3 * nc + cell] += mu * (v[2] - w2);
            tally[4 * nc + cell] += mu * 0.5 * ((v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) - (w0 * w0 + w1 * w1 + w2 * w2));
            v[0] = w0;
            v[1] = w1;
            v[2] = w2;
            I = 0.0;
            ksi = -std::log(1.0 - rng.uniform());
            ++nex;
        }
        if (kind == 1 || kind == 2) ++lost;
        if (trace) {
            double* r = trace + 8 * pid;
            r[0] = x[0];
            r[1] = x[1];
            r[2] = x[2];
            r[3] = v[0];
            r[4] = v[1];
            r[5] = v[2];
            r[6] = (double)nex;
            r[7] = 4.0 * (double)(visit + (kind == 0 || kind == 3 ? 1 : 0)) + (double)kind;
        }
    }
    for (int64_t c = 0; c < nc; ++c)
        for (int k = 0; k < 5; ++k) tally[k * nc + c] /= vol[c];
    if (ft)  // per unit face area; leaves also per box volume and centre x (Normir_velocity_volume)
        for (int64_t t = 0; t < ft->nface; ++t) {
            const double squ = fa[ft->face[t]];
            for (int k = 0; k < 3; ++k) ft->moments[3 * t + k] /= squ;
            for (int64_t l = ft->leaf_ptr[t]; l < ft->leaf_ptr[t + 1]; ++l) {
                const double* b = ft->leaf_box + 6 * l;
                ft->leaf_f[l] /= ((b[1] - b[0]) * (b[3] - b[2]) * (b[5] - b[4]) * squ * ((b[0] + b[1]) / 2.0));
            }
        }
    *lost_out = lost;
    return 0;
}

}  // extern "C"
