// Launch-shape dispatch of the face-flux kernel, shared by the translation
// units that instantiate it (FP64 / FP32 Riemann arithmetic, first / second
// order). The flux records are FP64 in every mode: the flux times area is
// part of the conservative accumulation.
#pragma once
#include "launch.h"
#include "step_kernels.cuh"

namespace titan {

template <typename R, int NK, bool MOVE, bool TVD>
static cudaError_t face_flux_variant(const FaceArgs& a, int v, cudaStream_t s) {
    switch (v) {
#define TITAN_FACE_CASE(i)                                                                              \
    case i: {                                                                                         \
        constexpr FaceVariant fv = kFaceVariant[i];                                                   \
        face_flux_kernel<R, double, NK, MOVE, fv.block, fv.min_blocks, TVD>                           \
            <<<blocks_for(a.M.nface, fv.block), fv.block, 0, s>>>(a);                                 \
        break;                                                                                        \
    }
        TITAN_FACE_CASE(0)
        TITAN_FACE_CASE(1)
        TITAN_FACE_CASE(2)
        TITAN_FACE_CASE(3)
        TITAN_FACE_CASE(4)
        TITAN_FACE_CASE(5)
        TITAN_FACE_CASE(6)
#undef TITAN_FACE_CASE
        default:
            return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <typename R, bool TVD>
static cudaError_t face_flux_dispatch(const FaceArgs& a, int nk, bool move, int variant, cudaStream_t s) {
    if (nk == 0 && !move) return face_flux_variant<R, 0, false, TVD>(a, variant, s);
    if (nk == 0 && move) return face_flux_variant<R, 0, true, TVD>(a, variant, s);
    if (nk == 2 && !move) return face_flux_variant<R, 2, false, TVD>(a, variant, s);
    if (nk == 2 && move) return face_flux_variant<R, 2, true, TVD>(a, variant, s);
    return cudaErrorInvalidValue;
}

}  // namespace titan
