// Monte-Carlo neutral hydrogen on the plasma mesh: the source generator the
// closure is trained on and falls back to.
//
// Physics restated from TITAN's MK_fly_immit (TITAN/source/Setka_MK.cpp:1752-2314):
//  * a neutral flies straight through the cells; in a cell its charge-exchange
//    frequency is nu = rho_Th * uz * sigma(uz) / Kn, uz = Velosity_1(|v - V_p|, cp)
//    (the Maxwell-averaged relative speed, Setka_MK.cpp:40-50), cp = sqrt(2 p_Th / rho_Th),
//    sigma(u) = (1 - a2 ln u)^2 (Phys_param.h:177-180) (Setka_MK.cpp:1976-1988);
//  * the optical depth accumulates nu * dt until it reaches -ln(1 - xi);
//  * at a charge exchange the new neutral velocity is drawn from the local proton
//    Maxwellian weighted by u sigma(u), by the rejection scheme of
//    Setka::M_K_Change_Velosity (Setka_MK.cpp:2788-2852);
//  * rho_Th, p_Th from Phys_param::Plasma_components_1 (Phys_param.cpp:628-665) with the
//    cell type as zone (Setka_MK.cpp:1956), floored as at Setka_MK.cpp:1966-1967.
// Added here (the reference tallies only densities, Cell.cpp:1042-1085): the
// momentum and energy the plasma gains at each exchange, mu (v_old - v_new) and
// mu (|v_old|^2 - |v_new|^2) / 2, per unit time and volume.
//
// Launch: neutrals enter through the hard outer boundary faces from a drifting
// Maxwellian (density n_H, bulk velocity u_H, thermal speed cp_H), the number per
// face proportional to its inflow flux; each carries weight mu = total inflow
// per unit time / N, so sum(mu * time in cell) / V is the density.
// Random numbers: a counter-based generator (SplitMix64 finaliser over seed,
// particle id and draw counter), so a run is reproducible for any launch shape.
//
// A pass on the device: the inflow CDF over all faces (a deterministic scan),
// one 256-byte tracing record per cell (McCell), one thread per neutral over
// those records, and the division of the tallies by the cell volumes.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/titan_b200.h"
#include "launch.h"
#include "mc.h"
#include "step_kernels.cuh"

namespace titan {
namespace mc {

constexpr double kSqrtPi = 1.77245385;  // sqrtpi_ of TITAN/source/Header.h:94

struct Rng {
    unsigned long long key;
    unsigned long long ctr;
    __device__ double uniform() {
        // SplitMix64 finaliser (Steele, Lea, Flood 2014) of a counter: a value in (0, 1)
        unsigned long long z = key + 0x9E3779B97F4A7C15ull * (++ctr);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z = z ^ (z >> 31);
        return ((double)(z >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    }
};

// Velosity_1 (Setka_MK.cpp:40-50): mean relative speed of a neutral moving at u
// through protons of thermal speed cp.
__device__ __forceinline__ double velosity_1(double u, double cp) {
    if (u < 0.00001)
        return 2.0 * cp / kSqrtPi + 2.0 * u * u / (3.0 * cp * kSqrtPi) - u * u * u * u / (15.0 * cp * cp * cp * kSqrtPi);
    return exp(-u * u / (cp * cp)) * cp / kSqrtPi + (u + (cp * cp) / (2.0 * u)) * erf(u / cp);
}

__device__ __forceinline__ double sigma(double a2, double x) {
    const double s = 1.0 - a2 * log(x);
    return s * s;
}

using Args = McArgs;

__device__ void plasma_in_cell(const Args& a, int c, double& rho_th, double& cp, double V[3]) {
    const int nc = a.M.ncell;
    const double rho = a.state[c], p = a.state[4 * nc + c];
    const double Q = a.P.npassive ? a.state[8 * nc + c] : 0.0;
    const double rho_He = a.P.npassive ? a.state[9 * nc + c] : 0.0;
    V[0] = a.state[nc + c];
    V[1] = a.state[2 * nc + c];
    V[2] = a.state[3 * nc + c];
    (void)Q;
    // the Monte-Carlo passes the cell type as the zone (Setka_MK.cpp:1956)
    const int al = (a.M.cell_type[c] <= 2) ? 2 : 1;
    double r = -(kMeDmp * al * rho_He + 4.0 * (-rho + rho_He)) / (4.0 * (1.0 + kMeDmp));
    double pt = p * (4.0 * rho - (4.0 + al * kMeDmp) * rho_He) / (8.0 * rho + (-7.0 + al + (1.0 - al) * kMeDmp) * rho_He);
    if (r <= 1e-8) r = 1e-8;
    if (pt <= 1e-8 / 2.0) pt = 1e-8 / 2.0;
    rho_th = r;
    cp = sqrt(2.0 * pt / r);
}

// New neutral velocity after an exchange (Setka::M_K_Change_Velosity): Ur/U are
// the proton bulk and V the old neutral velocity, all in units of cp.
__device__ void change_velocity(Rng& rng, double a2, double cp, const double U[3], const double Vn[3], double W[3]) {
    const double X = sqrt((Vn[0] - U[0]) * (Vn[0] - U[0]) + (Vn[1] - U[1]) * (Vn[1] - U[1]) +
                          (Vn[2] - U[2]) * (Vn[2] - U[2]));
    const double p4 = 0.5 * kSqrtPi * X / (1.0 + 0.5 * kSqrtPi * X);
    double v1 = U[0], v2 = U[1], v3 = U[2];
    for (int it = 0; it < 1000; ++it) {
        const double k1 = rng.uniform(), k2 = rng.uniform(), k3 = rng.uniform();
        const double k4 = rng.uniform(), k5 = rng.uniform(), k6 = rng.uniform();
        double y1, y2, y3;
        if (p4 < k1) {
            const double om1 = 1.0 - 2.0 * k4;
            const double so = sqrt(1.0 - om1 * om1);
            const double om2 = so * cos(2.0 * kPi * k5), om3 = so * sin(2.0 * kPi * k5);
            const double lo = sqrt(-log(k2 * k3));
            y1 = lo * om1;
            y2 = lo * om2;
            y3 = lo * om3;
        } else {
            y1 = sqrt(-log(k2)) * cos(kPi * k3);
            y2 = sqrt(-log(k4)) * cos(2.0 * kPi * k5);
            y3 = sqrt(-log(k4)) * sin(2.0 * kPi * k5);
        }
        v1 = y1 + U[0];
        v2 = y2 + U[1];
        v3 = y3 + U[2];
        const double u1 = Vn[0] - v1, u2 = Vn[1] - v2, u3 = Vn[2] - v3;
        const double uuu = sqrt(u1 * u1 + u2 * u2 + u3 * u3);
        const double yy = sqrt(y1 * y1 + y2 * y2 + y3 * y3);
        const double h = (uuu * sigma(a2, uuu * cp)) / (sigma(a2, X * cp) * (X + yy));
        if (!(h < k6)) break;
    }
    W[0] = v1;
    W[1] = v2;
    W[2] = v3;
}

// ---- inflow CDF over all faces, summed in a fixed order ----

constexpr double kSqrtPiFull = 1.7724538509055160273;  // sqrt(pi)

// Neutral inflow through face f per unit time: the flux of the drifting
// Maxwellian through the inward normal, n [cp e^{-s^2} / (2 sqrt(pi)) + u_n (1 + erf s) / 2]
// with s = u_n / cp, times the face area; 0 for faces that let no neutrals in.
__device__ __forceinline__ double inflow_weight(const Args& a, int f) {
    if (a.fd.index) {  // a tabulated face: its table's inflow (AMR_f::Culk_SpotokV)
        const int d = a.fd.index[f];
        if (d >= 0) return a.fd.flux[d] * a.L.fa[f];
    }
    const int t = a.M.face_type[f];
    if (t <= 0 || t > 31 || !((a.face_types >> t) & 1u)) return 0.0;
    const int nf = a.M.nface;
    const double un = -(a.uH0 * a.L.fn[f] + a.uH1 * a.L.fn[nf + f] + a.uH2 * a.L.fn[2 * nf + f]);
    const double sr = un / a.cpH;
    const double flux = a.nH * (a.cpH * exp(-sr * sr) / (2.0 * kSqrtPiFull) + 0.5 * un * (1.0 + erf(sr)));
    return flux * a.L.fa[f];
}

// Inclusive scan of v over a block of NT threads in a fixed order (warp shuffles,
// then the warp totals in ascending order); *all = the block total.
template <int NT>
__device__ __forceinline__ double block_scan(double v, double* warp_tot, double* all) {
    constexpr int kW = NT / 32;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double u = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += u;
    }
    if (lane == 31) warp_tot[w] = v;
    __syncthreads();
    double before = 0.0, sum = 0.0;
    for (int k = 0; k < kW; ++k) {
        if (k < w) before += warp_tot[k];
        sum += warp_tot[k];
    }
    __syncthreads();  // warp_tot is reused by the next call
    *all = sum;
    return before + v;
}

constexpr int kScanThreads = 256;
static_assert(kMcScanChunk % kScanThreads == 0, "whole rounds per block");

// Per block of kMcScanChunk faces: the inclusive prefix of the weights within
// the block into cdf, the block's total into block_sums.
__global__ void __launch_bounds__(kScanThreads) inflow_scan_kernel(Args a, double* cdf, double* block_sums) {
    __shared__ double warp_tot[kScanThreads / 32];
    const long long nf = a.M.nface;
    const long long base = (long long)blockIdx.x * kMcScanChunk;
    double carry = 0.0;
    for (int r = 0; r < kMcScanChunk / kScanThreads; ++r) {
        const long long f = base + r * kScanThreads + threadIdx.x;
        const double w = (f < nf) ? inflow_weight(a, (int)f) : 0.0;
        double all;
        const double incl = block_scan<kScanThreads>(w, warp_tot, &all);
        if (f < nf) cdf[f] = carry + incl;
        carry += all;
    }
    if (threadIdx.x == 0) block_sums[blockIdx.x] = carry;
}

// One block: block_sums[b] becomes the sum of the blocks before b, *total the sum
// of all. Each thread runs over a contiguous segment of the blocks.
constexpr int kBlockScanThreads = 1024;
__global__ void __launch_bounds__(kBlockScanThreads) inflow_blocks_kernel(double* block_sums, int nb,
                                                                         double* total) {
    __shared__ double warp_tot[kBlockScanThreads / 32];
    const int per = (nb + kBlockScanThreads - 1) / kBlockScanThreads;
    const int b0 = min(nb, (int)threadIdx.x * per), b1 = min(nb, b0 + per);
    double seg = 0.0;
    for (int b = b0; b < b1; ++b) {
        const double v = block_sums[b];
        block_sums[b] = seg;  // exclusive within the segment
        seg += v;
    }
    double all;
    const double before = block_scan<kBlockScanThreads>(seg, warp_tot, &all) - seg;
    for (int b = b0; b < b1; ++b) block_sums[b] += before;
    if (threadIdx.x == 0) *total = all;
}

// cdf[f] = (prefix within the block + blocks before) / total; the last entry is 1.
__global__ void inflow_finish_kernel(double* cdf, const double* block_sums, const double* total, int nf) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    const double T = *total;
    if (!(T > 0.0)) return;  // no inflow: the host reports it
    cdf[f] = (f == nf - 1) ? 1.0 : (cdf[f] + block_sums[f / kMcScanChunk]) / T;
}

// The tracing records of all cells (McCell): outward face planes in the
// cell's face order, neighbours, and the proton fluid of plasma_in_cell.
__global__ void pack_kernel(Args a, McCell* __restrict__ cells) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const MeshView& M = a.M;
    const int nc = M.ncell, nf = M.nface;
    if (c >= nc) return;
    McCell R;
#pragma unroll
    for (int sl = 0; sl < 6; ++sl) {
        const int fs = M.cell_faces[sl * nc + c];
        const int f = fs & 0x7fffffff;
        const double sg = (fs < 0) ? -1.0 : 1.0;  // outward normal of this cell
        const double n0 = sg * a.L.fn[f], n1 = sg * a.L.fn[nf + f], n2 = sg * a.L.fn[2 * nf + f];
        R.plane[sl][0] = n0;
        R.plane[sl][1] = n1;
        R.plane[sl][2] = n2;
        R.plane[sl][3] = a.L.fc[f] * n0 + a.L.fc[nf + f] * n1 + a.L.fc[2 * nf + f] * n2;
        R.nbr[sl] = (fs < 0) ? M.face_c0[f] : M.face_c1[f];
        if (a.ft.index) {  // a tallied face, reached from the table's side: the neutral stops there
            const int t = a.ft.index[f];
            if (t >= 0 && a.ft.side[t] == ((fs < 0) ? 1 : 0)) R.nbr[sl] = -3 - t;
        }
    }
    plasma_in_cell(a, c, R.rho_th, R.cp, R.V);
    cells[c] = R;
}

// A neutral that stops on tallied face table t (AMR_f::Add_particle,
// AMR_f.cpp:240-316): the moments mu / |v_n|, mu, mu / v_n^2, then its local
// velocity, clamped 1e-7 inside the table's bounds, adds mu to the first leaf
// that holds it (half-open boxes, the order of the table); where no leaf does,
// the point shrinks toward the origin by 0.995 and is looked up again, as the
// reference does, and after 30 tries counts as unplaced.
__device__ void tally_outgoing(const Args& a, int t, const double v[3]) {
    const McFaceTally& T = a.ft;
    const double* E = T.frame + 9 * (size_t)t;
    const double Vnn = fabs(v[0] * E[0] + v[1] * E[1] + v[2] * E[2]);
    atomicAdd(&T.mom[3 * t], a.mu / Vnn);
    atomicAdd(&T.mom[3 * t + 1], a.mu);
    atomicAdd(&T.mom[3 * t + 2], a.mu * ((1.0 / Vnn) * (1.0 / Vnn)));
    double x = v[0] * E[0] + v[1] * E[1] + v[2] * E[2];
    double y = v[0] * E[3] + v[1] * E[4] + v[2] * E[5];
    double z = v[0] * E[6] + v[1] * E[7] + v[2] * E[8];
    const double* B = T.bounds + 6 * (size_t)t;
    if (x < B[0]) x = B[0] + 1e-7;
    if (x > B[1]) x = B[1] - 1e-7;
    if (y < B[2]) y = B[2] + 1e-7;
    if (y > B[3]) y = B[3] - 1e-7;
    if (z < B[4]) z = B[4] + 1e-7;
    if (z > B[5]) z = B[5] - 1e-7;
    const int l0 = T.leaf_ptr[t], l1 = T.leaf_ptr[t + 1];
    for (int kk = 1; kk <= 30; ++kk) {
        for (int l = l0; l < l1; ++l) {
            const double* b = T.box + 6 * (size_t)l;
            if (b[0] <= x && x < b[1] && b[2] <= y && y < b[3] && b[4] <= z && z < b[5]) {
                atomicAdd(&T.f[l], a.mu);
                return;
            }
        }
        x *= 0.995;
        if (kk < 20) {
            y *= 0.995;
            z *= 0.995;
        }
    }
    atomicAdd(T.unplaced, 1ull);
}

__global__ void __launch_bounds__(128) trace_cells_kernel(Args a, const McCell* __restrict__ cells) {
    const long long pid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (pid >= a.nparticles) return;
    const MeshView& M = a.M;
    const int nc = M.ncell, nf = M.nface;
    Rng rng{a.seed ^ (0xD1B54A32D192ED03ull * (unsigned long long)(pid + 1)), 0ull};
    // stratified choice of the inflow face by its share of the flux (faces that
    // let no neutrals in add nothing to the CDF, so are never chosen)
    const double s = ((double)pid + rng.uniform()) / (double)a.nparticles;
    int lo = 0, hi = nf - 1;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a.inflow_cdf[mid] < s)
            lo = mid + 1;
        else
            hi = mid;
    }
    const int f0 = lo;
    // position: uniform on the quad (two triangles by area)
    double P[4][3];
#pragma unroll
    for (int k = 0; k < 4; ++k) load_node(a.L.xyz, M.nnode, M.face_nodes[k * nf + f0], P[k]);
    const double A1 = tri_area(P[0][0], P[0][1], P[0][2], P[1][0], P[1][1], P[1][2], P[2][0], P[2][1], P[2][2]);
    const double A2 = tri_area(P[0][0], P[0][1], P[0][2], P[3][0], P[3][1], P[3][2], P[2][0], P[2][1], P[2][2]);
    const int tb = (rng.uniform() * (A1 + A2) < A1) ? 1 : 3;
    double b1 = rng.uniform(), b2 = rng.uniform();
    if (b1 + b2 > 1.0) {
        b1 = 1.0 - b1;
        b2 = 1.0 - b2;
    }
    double x[3];
    for (int k = 0; k < 3; ++k) x[k] = P[0][k] + b1 * (P[tb][k] - P[0][k]) + b2 * (P[2][k] - P[0][k]);
    const int tab = a.fd.index ? a.fd.index[f0] : -1;
    double v[3] = {a.uH0, a.uH1, a.uH2};
    int cell = M.face_c0[f0];
    if (tab >= 0) {
        // velocity from the face's table: a leaf by its share of the inflow,
        // then the flux-weighted normal component and uniform tangential ones
        // in the leaf's box, turned into the face's frame
        const double u = rng.uniform();
        int l = a.fd.leaf_ptr[tab], h = a.fd.leaf_ptr[tab + 1] - 1;
        while (l < h) {
            const int mid = (l + h) >> 1;
            if (a.fd.cum[mid] < u)
                l = mid + 1;
            else
                h = mid;
        }
        const double* B = a.fd.box + 6 * (size_t)l;
        const double xL = B[0], xR = B[1];
        const double w0 = sqrt(xL * xL + rng.uniform() * (xR * xR - xL * xL));
        const double w1 = B[2] + rng.uniform() * (B[3] - B[2]);
        const double w2 = B[4] + rng.uniform() * (B[5] - B[4]);
        const double* E = a.fd.frame + 9 * (size_t)tab;
#pragma unroll
        for (int k = 0; k < 3; ++k) v[k] = w0 * E[k] + w1 * E[3 + k] + w2 * E[6 + k];
        if (a.fd.side[tab]) cell = M.face_c1[f0];
    }
    // velocity: flux-weighted drifting Maxwellian through the inward normal
    const double nin[3] = {-a.L.fn[f0], -a.L.fn[nf + f0], -a.L.fn[2 * nf + f0]};
    const double un = a.uH0 * nin[0] + a.uH1 * nin[1] + a.uH2 * nin[2];
    const double vmax = fmax(un, 0.0) + 6.0 * a.cpH;
    for (int it = 0; it < 4096 && tab < 0; ++it) {
        // Box-Muller pairs for exp(-y^2) per component
        const double r1 = sqrt(-log(rng.uniform())), t1 = 2.0 * kPi * rng.uniform();
        const double r2 = sqrt(-log(rng.uniform())), t2 = 2.0 * kPi * rng.uniform();
        v[0] = a.uH0 + a.cpH * r1 * cos(t1);
        v[1] = a.uH1 + a.cpH * r1 * sin(t1);
        v[2] = a.uH2 + a.cpH * r2 * cos(t2);
        const double vn = v[0] * nin[0] + v[1] * nin[1] + v[2] * nin[2];
        if (vn > 0.0 && rng.uniform() * vmax < vn) break;
    }
    double ksi = -log(1.0 - rng.uniform());
    double I = 0.0;
    double* T = a.tally;
    int nex = 0, visit = 0, kind = 1;  // end kind: 0 left, 1 lost, 2 no outgoing face
    for (; visit < a.max_cells; ++visit) {
        // the cell's record: its face planes, neighbours and proton fluid; the
        // ray leaves through the face it reaches first
        const McCell* R = cells + cell;
        double t_exit = 1e300;
        int next = -2;
#pragma unroll
        for (int sl = 0; sl < 6; ++sl) {
            const double2 nab = __ldg(reinterpret_cast<const double2*>(R->plane[sl]));
            const double2 ncd = __ldg(reinterpret_cast<const double2*>(R->plane[sl]) + 1);
            const double vn = v[0] * nab.x + v[1] * nab.y + v[2] * ncd.x;
            if (vn <= 0.0) continue;
            const double d = ncd.y - (x[0] * nab.x + x[1] * nab.y + x[2] * ncd.x);
            const double t = fmax(d, 0.0) / vn;
            if (t < t_exit) {
                t_exit = t;
                next = __ldg(R->nbr + sl);
            }
        }
        if (next == -2) {  // no outgoing face (degenerate): give up on this particle
            kind = 2;
            break;
        }
        const double rho_th = __ldg(&R->rho_th), cp = __ldg(&R->cp);
        const double Vp[3] = {__ldg(R->V), __ldg(R->V + 1), __ldg(R->V + 2)};
        const double du0 = v[0] - Vp[0], du1 = v[1] - Vp[1], du2 = v[2] - Vp[2];
        const double u = sqrt(du0 * du0 + du1 * du1 + du2 * du2);
        const double uz = velosity_1(u, cp);
        const double nu = rho_th * uz * sigma(a.P.par_a_2, uz) / a.P.par_Kn;
        const double dI = nu * t_exit;
        if (I + dI < ksi) {
            atomicAdd(&T[cell], a.mu * t_exit);
            I += dI;
            for (int k = 0; k < 3; ++k) x[k] += t_exit * v[k];
            if (next < 0) {  // left through the boundary, or stopped on a tallied face
                kind = 0;
                if (next <= -3) {
                    tally_outgoing(a, -3 - next, v);
                    kind = 3;
                }
                break;
            }
            cell = next;
            continue;
        }
        // charge exchange inside this cell
        const double t_ex = (ksi - I) / nu;
        atomicAdd(&T[cell], a.mu * t_ex);
        for (int k = 0; k < 3; ++k) x[k] += t_ex * v[k];
        const double U[3] = {Vp[0] / cp, Vp[1] / cp, Vp[2] / cp};
        const double Vn[3] = {v[0] / cp, v[1] / cp, v[2] / cp};
        double W[3];
        change_velocity(rng, a.P.par_a_2, cp, U, Vn, W);
        const double w0 = W[0] * cp, w1 = W[1] * cp, w2 = W[2] * cp;
        atomicAdd(&T[nc + cell], a.mu * (v[0] - w0));
        atomicAdd(&T[2 * nc + cell], a.mu * (v[1] - w1));
        atomicAdd(&T[3 * nc + cell], a.mu * (v[2] - w2));
        atomicAdd(&T[4 * nc + cell],
                  a.mu * 0.5 * ((v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) - (w0 * w0 + w1 * w1 + w2 * w2)));
        v[0] = w0;
        v[1] = w1;
        v[2] = w2;
        I = 0.0;
        ksi = -log(1.0 - rng.uniform());
        ++nex;
    }
    if (kind == 1 || kind == 2) atomicAdd(a.lost, 1ull);
    if (a.trace) {
        double* r = a.trace + 8 * pid;
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

// Divides the tallies by the cell volumes: n_H and the source densities.
__global__ void normalise_kernel(double* T, const double* vol, int nc) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    const double V = vol[c];
#pragma unroll
    for (int k = 0; k < 5; ++k) T[k * nc + c] /= V;
}

// The outgoing tables per unit face area; each leaf's weight also per unit box
// volume and box-centre normal speed (AMR_f::Normir_velocity_volume,
// AMR_f.cpp:318-336). One thread per table.
__global__ void tally_normalise_kernel(Args a, int ntab) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntab) return;
    const McFaceTally& T = a.ft;
    const double squ = a.L.fa[T.face[t]];
    for (int k = 0; k < 3; ++k) T.mom[3 * t + k] /= squ;
    for (int l = T.leaf_ptr[t]; l < T.leaf_ptr[t + 1]; ++l) {
        const double* b = T.box + 6 * (size_t)l;
        T.f[l] /= ((b[1] - b[0]) * (b[3] - b[2]) * (b[5] - b[4]) * squ * ((b[0] + b[1]) / 2.0));
    }
}

}  // namespace mc

cudaError_t launch_mc_tally_normalise(const McArgs& a, int ntab, cudaStream_t s) {
    mc::tally_normalise_kernel<<<blocks_for(ntab, 128), 128, 0, s>>>(a, ntab);
    return cudaGetLastError();
}

cudaError_t launch_mc_inflow_cdf(const McArgs& a, double* cdf, double* block_sums, double* total_out,
                                 cudaStream_t s) {
    const int nb = mc_scan_blocks(a.M.nface);
    mc::inflow_scan_kernel<<<nb, mc::kScanThreads, 0, s>>>(a, cdf, block_sums);
    mc::inflow_blocks_kernel<<<1, mc::kBlockScanThreads, 0, s>>>(block_sums, nb, total_out);
    mc::inflow_finish_kernel<<<blocks_for(a.M.nface, 256), 256, 0, s>>>(cdf, block_sums, total_out, a.M.nface);
    return cudaGetLastError();
}

cudaError_t launch_mc_pack(const McArgs& a, McCell* cells, cudaStream_t s) {
    mc::pack_kernel<<<blocks_for(a.M.ncell, 256), 256, 0, s>>>(a, cells);
    return cudaGetLastError();
}

cudaError_t launch_mc_trace_cells(const McArgs& a, const McCell* cells, cudaStream_t s) {
    mc::trace_cells_kernel<<<blocks_for(a.nparticles, 128), 128, 0, s>>>(a, cells);
    return cudaGetLastError();
}

cudaError_t launch_mc_normalise(double* tally, const double* vol, int ncell, cudaStream_t s) {
    mc::normalise_kernel<<<blocks_for(ncell, 256), 256, 0, s>>>(tally, vol, ncell);
    return cudaGetLastError();
}

}  // namespace titan
