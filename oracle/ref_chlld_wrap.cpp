// ORACLE / TEST INFRASTRUCTURE ONLY. Never linked into the shipped library.
//
// extern "C" wrapper around the reference's own Riemann solver
// `Phys_param::chlld` (TITAN/source/Phys_param.cpp:882-1878), which the
// recipe in oracle/Makefile compiles unmodified from the reference tree into
// oracle/_ref/libtitan_ref.so. Tests and the golden-vector generator call it
// through ctypes to pin the oracle's restatement and the CUDA kernels.
#include "Phys_param.h"

#include <unistd.h>

// TITAN/source/Help_funk.cpp:219-232 — orthonormal (t, m) completing n.
void get_bazis(const Eigen::Vector3d& n, Eigen::Vector3d& t, Eigen::Vector3d& m) {
    Eigen::Vector3d a(1.0, 0.0, 0.0);
    if (std::abs(n.dot(a)) > 0.9) a = Eigen::Vector3d(0.0, 1.0, 0.0);
    t = a.cross(n).normalized();
    m = n.cross(t);
}

// TITAN/source/Help_funk.cpp:244-249.
double scalarProductFast(const double& ax, const double& ay, const double& az,
                         const double& bx, const double& by, const double& bz) {
    return ax * bx + ay * by + az * bz;
}

static Phys_param* g_param = nullptr;

extern "C" {

// Constructs the reference's Phys_param. Its constructor reads
// set_parameters.txt, set_model_parameters.txt and nVT1au_new_2000-2022av.dat
// from the current directory (Phys_param.cpp:339-370, :545-622), so this
// switches into `run_dir` (written by the recipe) for the duration.
int titan_ref_init(const char* run_dir) {
    if (g_param) return 0;
    char old[4096];
    if (!getcwd(old, sizeof(old))) return -1;
    if (chdir(run_dir) != 0) return -2;
    g_param = new Phys_param();
    if (chdir(old) != 0) return -3;
    return 0;
}

void titan_ref_set_gamma(double gamma) {
    g_param->gamma = gamma;
    g_param->g1 = gamma - 1.0;
}

// One call of the reference solver. q1/q2: (rho,u,v,w,p,Bx,By,Bz) with
// Gaussian B; qout: 8 fluxes; kl/kr/kout: n_k passive scalars; ds: dsl,dsc,dsr.
void titan_ref_chlld(int n_state, const double* nrm, double w, const double* q1,
                     const double* q2, int null_bn, int n_disc, int n_k,
                     const double* kl, const double* kr, double* qout, double* kout,
                     double* ds, int left_ydar, int contact) {
    std::vector<double> qqq1(q1, q1 + 8), qqq2(q2, q2 + 8), qqq(8, 0.0);
    std::vector<double> KL(kl, kl + n_k), KR(kr, kr + n_k), K(n_k, 0.0);
    double dsr = 0, dsc = 0, dsl = 0;
    PrintOptions opt{};
    g_param->chlld((unsigned short)n_state, nrm[0], nrm[1], nrm[2], w, qqq1, qqq2, qqq,
                   null_bn != 0, (unsigned short)n_disc, KL, KR, K, dsr, dsc, dsl, opt,
                   left_ydar != 0, contact != 0);
    for (int i = 0; i < 8; ++i) qout[i] = qqq[i];
    for (int i = 0; i < n_k; ++i) kout[i] = K[i];
    ds[0] = dsl;
    ds[1] = dsc;
    ds[2] = dsr;
}

// One call of the reference's exact gas-dynamic Godunov solver used on HP
// faces with bn_in_p_on_HP (Phys_param::Godunov_Solver_Alexashov,
// Phys_param.cpp:1938-2385). q1/q2: (rho,u,v,w,p,...); qout: 5 fluxes
// (mass, momentum, energy); ds: dsl, dsc, dsr. The reference exits on
// inputs its Newton iterations cannot handle; callers pass valid states.
void titan_ref_godunov(const double* nrm, double w, const double* q1, const double* q2, int contact,
                       double* qout, double* ds) {
    std::vector<double> qqq1(q1, q1 + 8), qqq2(q2, q2 + 8), qqq(8, 0.0), n(nrm, nrm + 3);
    double dsl = 0, dsp = 0, dsc = 0;
    g_param->Godunov_Solver_Alexashov(qqq1, qqq2, n, qqq, dsl, dsp, dsc, w, contact != 0);
    for (int i = 0; i < 5; ++i) qout[i] = qqq[i];
    ds[0] = dsl;
    ds[1] = dsc;
    ds[2] = dsp;
}

// Batched form: n faces, arrays of stride 8 (states/fluxes) and 3 (normals, ds).
void titan_ref_chlld_batch(long n, const int* n_state, const double* nrm, const double* w,
                           const double* q1, const double* q2, double* qout, double* ds) {
    for (long i = 0; i < n; ++i) {
        double dummy = 0.0;
        titan_ref_chlld(n_state[i], nrm + 3 * i, w[i], q1 + 8 * i, q2 + 8 * i, 0, 0, 0,
                        &dummy, &dummy, qout + 8 * i, &dummy, ds + 3 * i, 0, 0);
    }
}

// TITAN/source/Phys_param.cpp:826-874 (exact flux of one state through n).
void titan_ref_get_potok(const double* q, const double* nrm, double* potok) {
    std::vector<double> P(8, 0.0);
    g_param->Get_Potok(q[0], q[4], q[1], q[2], q[3], q[5], q[6], q[7], nrm[0], nrm[1], nrm[2], P);
    for (int i = 0; i < 8; ++i) potok[i] = P[i];
}

// TITAN/source/Phys_param.cpp:628-665 — thermal-proton split.
void titan_ref_plasma_components_1(int zone, double rho, double p, double rho_he,
                                   double* out3) {
    std::unordered_map<std::string, double> cell, par;
    cell["rho"] = rho;
    cell["p"] = p;
    cell["rho_He"] = rho_he;
    g_param->Plasma_components_1((short)zone, cell, par);
    out3[0] = par["rho_Th"];
    out3[1] = par["p_Th"];
    out3[2] = par["T_Th"];
}

}  // extern "C"
