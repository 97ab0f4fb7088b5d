// Cell-update translation unit (-fmad=false, like kernels_fp64.cu): the
// per-cell gather of face fluxes, the conservative update with sources and
// floors, the next layer's cell geometry, and the CFL rollover.
#include "closure.h"
#include "launch.h"
#include "step_kernels.cuh"

namespace titan {

template <typename FT, int NK, bool MOVE, int SRC, int BS, int MINB>
__global__ void __launch_bounds__(BS, MINB) cell_update_kernel(CellArgs a) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const bool ok = a.st->err_kind == 0;
    if (c < a.M.ncell && ok) {
        const MeshView& M = a.M;
        const int nc = M.ncell;
        const double time = a.st->dt;
        const double Volume = a.vol1[c];
        double Volume2 = Volume;
        double C2[3] = {0.0, 0.0, 0.0};
        if (MOVE) {
            // centre and volume of the next layer (Cell::Culc_center / Culc_volume);
            // stored after the gather, so the stores do not hold its loads back
            const int nn = M.nnode;
            double X[8][3];
#pragma unroll
            for (int k = 0; k < 8; ++k) load_node(a.L2.xyz, nn, M.cell_nodes[k * nc + c], X[k]);
            cell_centre(X, C2);
            Volume2 = cell_volume(C2, [&](int s, int k, double* p) {
                const int li = (M.cell_fmap[s * nc + c] >> (3 * k)) & 7;
                load_node(a.L2.xyz, nn, M.cell_nodes[li * nc + c], p);
            });
        }
        using L = FluxLayout<FT, NK>;
        double PO[9 + NK];
#pragma unroll
        for (int k = 0; k < 9 + NK; ++k) PO[k] = 0.0;
        const FT* fx = reinterpret_cast<const FT*>(a.flux);
#pragma unroll
        for (int s = 0; s < 6; ++s) {
            const int fs = M.cell_faces[s * nc + c];
            const int f = fs & 0x7fffffff;
            const double sign = (fs < 0) ? -1.0 : 1.0;
            const FT* src = fx + size_t(f) * L::stride;
            FT v[L::stride];
            if (sizeof(FT) == 8) {
#pragma unroll
                for (int k = 0; k < L::stride; k += 2) {
                    const double2 t = __ldg(reinterpret_cast<const double2*>(src) + k / 2);
                    v[k] = FT(t.x);
                    v[k + 1] = FT(t.y);
                }
            } else {
#pragma unroll
                for (int k = 0; k < L::stride; k += 4) {
                    const float4 t = __ldg(reinterpret_cast<const float4*>(src) + k / 4);
                    v[k] = FT(t.x);
                    v[k + 1] = FT(t.y);
                    v[k + 2] = FT(t.z);
                    v[k + 3] = FT(t.w);
                }
            }
#pragma unroll
            for (int k = 0; k < 9 + NK; ++k) PO[k] += sign * double(v[k]);
        }
        double prim[NV];
#pragma unroll
        for (int k = 0; k < 8 + NK; ++k) prim[k] = a.state[k * nc + c];
#pragma unroll
        for (int k = 8 + NK; k < NV; ++k) prim[k] = 0.0;
        if (MOVE) {
            a.L2.cc[c] = C2[0];
            a.L2.cc[nc + c] = C2[1];
            a.L2.cc[2 * nc + c] = C2[2];
            a.L2.vol[c] = Volume2;
        }
        double S[4] = {0.0, 0.0, 0.0, 0.0};
        if (SRC == 1) {
            bera_sources(a.P, prim, M.cell_type[c], a.hfl, nc, c, S);
        } else if (SRC == 2) {
#pragma unroll
            for (int k = 0; k < 4; ++k) S[k] = a.src[k * nc + c];
        } else if (SRC == 3) {
            // the closure's sources for this step's state, in its frame at the current centre
            const ClosureCell& q = a.cl;
            const bool out_env = q.outside[c] != 0;
            if (out_env && q.fallback) {
#pragma unroll
                for (int k = 0; k < 4; ++k) S[k] = q.fallback[k * nc + c];
            } else {
                float y[5];
#pragma unroll
                for (int k = 0; k < 5; ++k) y[k] = q.y[k * nc + c];
                closure_sources(y, q.norm + 16, prim[0], prim[1], prim[2], prim[3], q.cc1[c], q.cc1[nc + c],
                                q.cc1[2 * nc + c], q.nH_inf, q.lambda, S);
            }
            if (out_env && q.n_outside) atomicAdd(q.n_outside, 1ull);
        }
        const double g1 = a.P.gamma - 1.0;
        const double cpi4 = 4.0 * kPi;
        const double rho = prim[0], vx = prim[1], vy = prim[2], vz = prim[3], p = prim[4];
        const double bx = prim[5], by = prim[6], bz = prim[7], Q = prim[8], rho_He = prim[9];
        const double dsk = vx * bx + vy * by + vz * bz;
        double rho3 = rho * Volume / Volume2 - time * PO[0] / Volume2;
        bool rho_null = false;
        if (rho3 < 1e-7) {
            rho_null = true;
            rho3 = 0.1;
            atomicAdd(&a.st->n_rho_floor, 1ull);
        }
        double Q3 = 0.0, rho_He3 = 0.0;
        if (NK > 0) {
            Q3 = Q * Volume / Volume2 - time * PO[9] / Volume2;
            rho_He3 = rho_He * Volume / Volume2 - time * PO[9 + (NK > 1 ? 1 : 0)] / Volume2;
        }
        if (rho_He3 < 0.0) rho_He3 = 0.0;
        double u3, v3, w3, bx3, by3, bz3, p3;
        if (!rho_null) {
            u3 = (rho * vx * Volume / Volume2 - time * (PO[1] + (bx / cpi4) * PO[8]) / Volume2 + time * S[0]) / rho3;
            v3 = (rho * vy * Volume / Volume2 - time * (PO[2] + (by / cpi4) * PO[8]) / Volume2 + time * S[1]) / rho3;
            w3 = (rho * vz * Volume / Volume2 - time * (PO[3] + (bz / cpi4) * PO[8]) / Volume2 + time * S[2]) / rho3;
            bx3 = bx * Volume / Volume2 - time * (PO[5] + vx * PO[8]) / Volume2;
            by3 = by * Volume / Volume2 - time * (PO[6] + vy * PO[8]) / Volume2;
            bz3 = bz * Volume / Volume2 - time * (PO[7] + vz * PO[8]) / Volume2;
            p3 = (((p / g1 + 0.5 * rho * (vx * vx + vy * vy + vz * vz) + (bx * bx + by * by + bz * bz) / kC8Pi) *
                       Volume / Volume2 -
                   time * (PO[4] + (dsk / cpi4) * PO[8]) / Volume2 + time * S[3]) -
                  0.5 * rho3 * (u3 * u3 + v3 * v3 + w3 * w3) - (bx3 * bx3 + by3 * by3 + bz3 * bz3) / kC8Pi) *
                 g1;
            if (M.cell_type[c] == 2) {  // Zone_2 effective magnetic dissipation, tau = 1
                const double tau = 1.0;
                const double bx4 = bx3 - time * bx3 / tau;
                const double by4 = by3 - time * by3 / tau;
                const double bz4 = bz3 - time * bz3 / tau;
                const double p4 = p3 + (time / tau - (time / tau) * (time / tau)) * (g1) *
                                           (bx3 * bx3 + by3 * by3 + bz3 * bz3) / (4.0 * kPi);
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
        if (isnan(rho3) || (rho3 != 0.0 && fabs(rho3) < 2.2250738585072014e-308) || isnan(Q3) ||
            (Q3 != 0.0 && fabs(Q3) < 2.2250738585072014e-308))
            record_error(a.st, 20, c);
        if (p3 < 0.00000001) {
            p3 = 0.000001;
            atomicAdd(&a.st->n_p_floor, 1ull);
        }
        if (rho_He3 > rho3) rho_He3 = rho3 * 0.1;
        double* o = a.state2;
        o[c] = rho3;
        o[nc + c] = u3;
        o[2 * nc + c] = v3;
        o[3 * nc + c] = w3;
        o[4 * nc + c] = p3;
        const bool tvd = M.cell_tvd[c] != 0;
        o[5 * nc + c] = tvd ? bx3 : bx;
        o[6 * nc + c] = tvd ? by3 : by;
        o[7 * nc + c] = tvd ? bz3 : bz;
        if (NK > 0) {
            o[8 * nc + c] = Q3;
            if (NK > 1) o[9 * nc + c] = rho_He3;
        }
        if (SRC == 3) {
            // the closure's inputs for the next step, from the state just written
            const ClosureCell& q = a.cl;
            float f[8];
            // the centre the next step's closure sees: the next layer's (moving mesh) or this one
            const double cx = MOVE ? C2[0] : q.cc1[c], cy = MOVE ? C2[1] : q.cc1[nc + c];
            const double cz = MOVE ? C2[2] : q.cc1[2 * nc + c];
            closure_features(rho3, u3, v3, w3, p3, cx, cy, cz, q.nH_inf, q.lambda, f);
            uint32_t w8[8];
            bool out = false;
            closure_words(f, q.norm, q.env, w8, out);
#pragma unroll
            for (int k = 0; k < 8; ++k) q.in[(size_t)k * nc + c] = w8[k];
            q.outside[c] = out ? 1 : 0;
        }
    }
    // Last block to finish rolls the clock: t += dt, dt = CFL minimum of this
    // step's faces (applied on the next step, Setka_physics.cpp:1606-1607).
    __shared__ bool last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned int prev = atomicAdd(&a.st->block_counter, 1u);
        last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        DevStatus* st = a.st;
        const unsigned long long bits = atomicAdd(&st->dt_next_bits, 0ull);
        if (st->err_kind == 0) {
            st->t += st->dt;
            st->dt = __longlong_as_double((long long)bits);
            st->steps_done += 1ull;
        }
        st->dt_next_bits = (unsigned long long)__double_as_longlong(100000000.0);
        st->block_counter = 0u;
        __threadfence();
    }
}

template <typename FT, int NK, bool MOVE, int BS, int MINB>
static void cell_update_src(const CellArgs& a, int src, cudaStream_t s) {
    const unsigned int g = blocks_for(a.M.ncell, BS);
    if (src == 0) cell_update_kernel<FT, NK, MOVE, 0, BS, MINB><<<g, BS, 0, s>>>(a);
    else if (src == 1) cell_update_kernel<FT, NK, MOVE, 1, BS, MINB><<<g, BS, 0, s>>>(a);
    else if (src == 2) cell_update_kernel<FT, NK, MOVE, 2, BS, MINB><<<g, BS, 0, s>>>(a);
    else cell_update_kernel<FT, NK, MOVE, 3, BS, MINB><<<g, BS, 0, s>>>(a);
}

template <typename FT, int NK, bool MOVE>
static cudaError_t cell_update_variant(const CellArgs& a, int src, int v, cudaStream_t s) {
    switch (v) {
#define TITAN_CELL_CASE(i)                                                                   \
    case i:                                                                                \
        cell_update_src<FT, NK, MOVE, kCellVariant[i].block, kCellVariant[i].min_blocks>(a, src, s); \
        break;
        TITAN_CELL_CASE(0)
        TITAN_CELL_CASE(1)
        TITAN_CELL_CASE(2)
        TITAN_CELL_CASE(3)
        TITAN_CELL_CASE(4)
        TITAN_CELL_CASE(5)
#undef TITAN_CELL_CASE
        default:
            return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_cell_update(const CellArgs& a, int nk, bool move, int src, int variant, cudaStream_t s) {
    if (nk == 0 && !move) return cell_update_variant<double, 0, false>(a, src, variant, s);
    if (nk == 0 && move) return cell_update_variant<double, 0, true>(a, src, variant, s);
    if (nk == 2 && !move) return cell_update_variant<double, 2, false>(a, src, variant, s);
    if (nk == 2 && move) return cell_update_variant<double, 2, true>(a, src, variant, s);
    return cudaErrorInvalidValue;
}

}  // namespace titan
