// Cell-update translation unit (-fmad=false, like kernels_fp64.cu): the
// per-cell gather of face fluxes, the conservative update with sources and
// floors, the next layer's cell geometry, and the CFL rollover.
#include "closure.h"
#include "launch.h"
#include "step_kernels.cuh"

namespace titan {

// The update of cell c. `gather(PO)` sums the cell's six face records into
// PO in the cell's own face order (the flux gather of Setka_physics.cpp:
// 1671-1733); the launch shapes differ only in where the records come from.
template <int NK, bool MOVE, int SRC, typename Gather>
__device__ __forceinline__ void update_cell(const CellArgs& a, const int c, Gather&& gather) {
    {
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
        double PO[9 + NK];
        gather(PO);
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
}

// Last block to finish rolls the clock: t += dt, dt = CFL minimum of this
// step's faces (applied on the next step, Setka_physics.cpp:1606-1607).
__device__ __forceinline__ void roll_clock(const CellArgs& a) {
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



// One face record (9 + NK fluxes times area, padded to 16 bytes) added into PO
// with the face's sign: from global memory through the read-only path, or from
// shared memory where the staged update put it.
template <int NK>
__device__ __forceinline__ void add_record_global(const double* src, double sign, double* PO) {
    constexpr int S = FluxLayout<double, NK>::stride;
    double v[S];
#pragma unroll
    for (int k = 0; k < S; k += 2) {
        const double2 t = __ldg(reinterpret_cast<const double2*>(src) + k / 2);
        v[k] = t.x;
        v[k + 1] = t.y;
    }
#pragma unroll
    for (int k = 0; k < 9 + NK; ++k) PO[k] += sign * v[k];
}

template <int NK>
__device__ __forceinline__ void add_record_shared(const double* src, double sign, double* PO) {
    constexpr int S = FluxLayout<double, NK>::stride;
    double v[S];
#pragma unroll
    for (int k = 0; k < S; k += 2) {
        const double2 t = reinterpret_cast<const double2*>(src)[k / 2];
        v[k] = t.x;
        v[k + 1] = t.y;
    }
#pragma unroll
    for (int k = 0; k < 9 + NK; ++k) PO[k] += sign * v[k];
}

// One thread per cell; each record is read from global memory where it is
// needed (two dependent loads per face: the face id, then the record).
template <int NK, bool MOVE, int SRC, int BS, int MINB>
__global__ void __launch_bounds__(BS, MINB) cell_update_kernel(CellArgs a) {
    const int c = blockIdx.x * BS + threadIdx.x;
    if (c < a.M.ncell && a.st->err_kind == 0) {
        update_cell<NK, MOVE, SRC>(a, c, [&](double* PO) {
            constexpr int S = FluxLayout<double, NK>::stride;
            const double* fx = static_cast<const double*>(a.flux);
            const int nc = a.M.ncell;
#pragma unroll
            for (int k = 0; k < 9 + NK; ++k) PO[k] = 0.0;
#pragma unroll
            for (int s = 0; s < 6; ++s) {
                const int fs = a.M.cell_faces[s * nc + c];
                add_record_global<NK>(fx + size_t(fs & 0x7fffffff) * S, fs < 0 ? -1.0 : 1.0, PO);
            }
        });
    }
    roll_clock(a);
}

// Shared memory of the staged update: an mbarrier, then the records of the
// faces the block's cells own (cells[0] in the block), at most `cap` of them
// (4.25 per cell; the renumbered shells need at most 4.2), then OV slots per
// thread for records of the cell's other faces.
template <int NK, int BS, int OV>
struct StagedSmem {
    static constexpr int S = FluxLayout<double, NK>::stride;
    static constexpr int cap = (17 * BS) / 4;
    static constexpr size_t bytes = 16 + sizeof(double) * S * (size_t(cap) + size_t(OV) * BS);
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Sleeping wait on phase 0 of an mbarrier: try_wait with a 100 us suspend
// hint, at most ~1 s (globaltimer) and 2^14 calls; false when it ran out.
__device__ __forceinline__ bool stage_wait(uint32_t mbar) {
    uint64_t t0;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
    for (int it = 0; it < (1 << 14); ++it) {
        uint32_t done = 0;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0, %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(100000u)
            : "memory");
        if (done) return true;
        uint64_t t;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        if (t - t0 > 1000000000ull) return false;
    }
    return false;
}

// The block's wait for its staged records. A wait that runs out records
// error kind 21 (the step then reports TITAN_ETIMEOUT) and waits once more,
// so the block does not leave while its copy may still be writing.
__device__ __forceinline__ void stage_wait_or_flag(uint32_t mbar, DevStatus* st, int index) {
    if (!stage_wait(mbar)) {
        record_error(st, 21, index);
        stage_wait(mbar);
    }
}

// The cell update with its face records staged in shared memory. Faces are
// sorted by cells[0], so the faces owned by the block's cells are one
// contiguous run of records: one elected thread copies it with a single bulk
// TMA copy (cp.async.bulk, completion counted on an mbarrier) while every
// thread gathers its cell's nodes, state and face ids. A record outside that
// run (a face whose owner is in another block, about one per cell on the
// shells) is copied by its thread with cp.async into its own slots, up to OV
// of them; any beyond are read from global memory. The sums run in the cell's
// own face order, as in cell_update_kernel, so results are identical.
template <int NK, bool MOVE, int SRC, int BS, int MINB, int OV>
__global__ void __launch_bounds__(BS, MINB) cell_update_staged_kernel(CellArgs a) {
    using SM = StagedSmem<NK, BS, OV>;
    constexpr int S = SM::S;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int go_s;
    double* stage = reinterpret_cast<double*>(smem + 16);
    double* ov = stage + size_t(SM::cap) * S;
    const uint32_t mbar = smem_addr(smem);
    const int nc = a.M.ncell;
    const int tid = threadIdx.x;
    const int cb = blockIdx.x * BS;
    const int c = cb + tid;
    const int nchunk = (nc + 31) >> 5;
    const int fb = a.owner_start[cb >> 5];
    const int fe = a.owner_start[min((cb + BS) >> 5, nchunk)];
    const int nstage = min(fe - fb, SM::cap);
    const double* fx = static_cast<const double*>(a.flux);
    if (tid == 0) {
        const int go = a.st->err_kind == 0;
        go_s = go;
        if (go && nstage > 0) {
            const uint32_t bytes = uint32_t(nstage) * S * sizeof(double);
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            asm volatile(
                "{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(mbar),
                "r"(bytes)
                : "memory");
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                    smem_addr(stage)),
                "l"(fx + size_t(fb) * S), "r"(bytes), "r"(mbar)
                : "memory");
        }
    }
    __syncthreads();
    const bool go = go_s != 0;
    const bool staged = go && nstage > 0;
    if (c < nc && go) {
        int fs[6];
#pragma unroll
        for (int s = 0; s < 6; ++s) fs[s] = a.M.cell_faces[s * nc + c];
        {
            int k = 0;
#pragma unroll
            for (int s = 0; s < 6; ++s) {
                const int f = fs[s] & 0x7fffffff;
                if ((unsigned)(f - fb) >= (unsigned)nstage && k < OV) {
                    const uint32_t dst = smem_addr(ov + size_t(k * BS + tid) * S);
                    const double* src = fx + size_t(f) * S;
#pragma unroll
                    for (int j = 0; j < S; j += 2)
                        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst + 8u * j), "l"(src + j)
                                     : "memory");
                    ++k;
                }
            }
        }
        update_cell<NK, MOVE, SRC>(a, c, [&](double* PO) {
            asm volatile("cp.async.wait_all;" ::: "memory");
            if (staged) stage_wait_or_flag(mbar, a.st, cb);
#pragma unroll
            for (int k = 0; k < 9 + NK; ++k) PO[k] = 0.0;
            int k = 0;
#pragma unroll
            for (int s = 0; s < 6; ++s) {
                const int f = fs[s] & 0x7fffffff;
                const double sign = fs[s] < 0 ? -1.0 : 1.0;
                if ((unsigned)(f - fb) < (unsigned)nstage) {
                    add_record_shared<NK>(stage + size_t(f - fb) * S, sign, PO);
                } else if (k < OV) {
                    add_record_shared<NK>(ov + size_t(k * BS + tid) * S, sign, PO);
                    ++k;
                } else {
                    add_record_global<NK>(fx + size_t(f) * S, sign, PO);
                }
            }
        });
    } else if (staged) {
        stage_wait_or_flag(mbar, a.st, cb);
    }
    roll_clock(a);
}

template <int NK, bool MOVE, int SRC, int BS, int MINB>
static cudaError_t plain_launch(const CellArgs* a, cudaStream_t s) {
    if (!a) return cudaSuccess;
    cell_update_kernel<NK, MOVE, SRC, BS, MINB><<<blocks_for(a->M.ncell, BS), BS, 0, s>>>(*a);
    return cudaGetLastError();
}

// The staged kernels need more than 48 KB of dynamic shared memory: with a
// null `a` this sets the attribute on the current device (cell_update_prepare,
// called when a context is created, so never while a stream is captured).
template <int NK, bool MOVE, int SRC, int BS, int MINB, int OV>
static cudaError_t staged_launch(const CellArgs* a, cudaStream_t s) {
    constexpr int bytes = (int)StagedSmem<NK, BS, OV>::bytes;
    if (!a)
        return cudaFuncSetAttribute(cell_update_staged_kernel<NK, MOVE, SRC, BS, MINB, OV>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (!a->owner_start) return cudaErrorInvalidValue;
    cell_update_staged_kernel<NK, MOVE, SRC, BS, MINB, OV><<<blocks_for(a->M.ncell, BS), BS, bytes, s>>>(*a);
    return cudaGetLastError();
}

template <int NK, bool MOVE, int BS, int MINB, int OV>
static cudaError_t variant_src(const CellArgs* a, int src, cudaStream_t s) {
    if constexpr (OV == 0) {
        if (src == 0) return plain_launch<NK, MOVE, 0, BS, MINB>(a, s);
        if (src == 1) return plain_launch<NK, MOVE, 1, BS, MINB>(a, s);
        if (src == 2) return plain_launch<NK, MOVE, 2, BS, MINB>(a, s);
        return plain_launch<NK, MOVE, 3, BS, MINB>(a, s);
    } else {
        if (src == 0) return staged_launch<NK, MOVE, 0, BS, MINB, OV>(a, s);
        if (src == 1) return staged_launch<NK, MOVE, 1, BS, MINB, OV>(a, s);
        if (src == 2) return staged_launch<NK, MOVE, 2, BS, MINB, OV>(a, s);
        return staged_launch<NK, MOVE, 3, BS, MINB, OV>(a, s);
    }
}

template <int NK, bool MOVE>
static cudaError_t cell_update_variant(const CellArgs* a, int src, int v, cudaStream_t s) {
    switch (v) {
#define TITAN_CELL_CASE(i)                                                                                   \
    case i:                                                                                                  \
        return variant_src<NK, MOVE, kCellVariant[i].block, kCellVariant[i].min_blocks, kCellVariant[i].overflow>( \
            a, src, s);
        TITAN_CELL_CASE(0)
        TITAN_CELL_CASE(1)
        TITAN_CELL_CASE(2)
        TITAN_CELL_CASE(3)
        TITAN_CELL_CASE(4)
        TITAN_CELL_CASE(5)
        TITAN_CELL_CASE(6)
        TITAN_CELL_CASE(7)
        TITAN_CELL_CASE(8)
#undef TITAN_CELL_CASE
        default:
            return cudaErrorInvalidValue;
    }
}

static cudaError_t cell_update_dispatch(const CellArgs* a, int nk, bool move, int src, int variant, cudaStream_t s) {
    if (nk == 0 && !move) return cell_update_variant<0, false>(a, src, variant, s);
    if (nk == 0 && move) return cell_update_variant<0, true>(a, src, variant, s);
    if (nk == 2 && !move) return cell_update_variant<2, false>(a, src, variant, s);
    if (nk == 2 && move) return cell_update_variant<2, true>(a, src, variant, s);
    return cudaErrorInvalidValue;
}

cudaError_t launch_cell_update(const CellArgs& a, int nk, bool move, int src, int variant, cudaStream_t s) {
    return cell_update_dispatch(&a, nk, move, src, variant, s);
}

cudaError_t cell_update_prepare() {
    for (int nk = 0; nk <= 2; nk += 2)
        for (int move = 0; move <= 1; ++move)
            for (int src = 0; src <= 3; ++src)
                for (int v = 0; v < kCellVariants; ++v) {
                    const cudaError_t e = cell_update_dispatch(nullptr, nk, move != 0, src, v, nullptr);
                    if (e) return e;
                }
    return cudaSuccess;
}

}  // namespace titan
