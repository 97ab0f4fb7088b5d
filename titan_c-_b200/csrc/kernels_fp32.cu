// FP32-flux translation unit: the Riemann flux in single precision (the
// mixed-precision step keeps reconstruction, accumulation, update and the CFL
// reduction in FP64). Contraction to FMA is allowed here, and single-precision
// division and square root use the fast approximate forms (-prec-div=false,
// -prec-sqrt=false): the flux error budget is 1e-4, far above their few ulp.
#include "launch.h"
#include "step_kernels.cuh"

namespace titan {

template <typename R, int NK, bool MOVE>
static cudaError_t face_flux_variant(const FaceArgs& a, int v, cudaStream_t s) {
    switch (v) {
#define TITAN_FACE_CASE(i)                                                                              \
    case i: {                                                                                         \
        constexpr FaceVariant fv = kFaceVariant[i];                                                   \
        face_flux_kernel<R, R, NK, MOVE, fv.block, fv.min_blocks>                                     \
            <<<blocks_for(a.M.nface, fv.block), fv.block, 0, s>>>(a);                                 \
        break;                                                                                        \
    }
        TITAN_FACE_CASE(0)
        TITAN_FACE_CASE(1)
        TITAN_FACE_CASE(2)
        TITAN_FACE_CASE(3)
        TITAN_FACE_CASE(4)
        TITAN_FACE_CASE(5)
#undef TITAN_FACE_CASE
        default:
            return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_face_flux_fp32(const FaceArgs& a, int nk, bool move, int variant, cudaStream_t s) {
    if (nk == 0 && !move) return face_flux_variant<float, 0, false>(a, variant, s);
    if (nk == 0 && move) return face_flux_variant<float, 0, true>(a, variant, s);
    if (nk == 2 && !move) return face_flux_variant<float, 2, false>(a, variant, s);
    if (nk == 2 && move) return face_flux_variant<float, 2, true>(a, variant, s);
    return cudaErrorInvalidValue;
}

cudaError_t launch_riemann_batch_fp32(long long n, const signed char* ns, const double* nrm, const double* w,
                                      const double* q1, const double* q2, double* flux, double* ds, int* rc,
                                      int flags, double gamma, cudaStream_t s) {
    riemann_batch_kernel<float><<<blocks_for(n, 128), 128, 0, s>>>(n, ns, nrm, w, q1, q2, flux, ds, rc, flags, gamma);
    return cudaGetLastError();
}

}  // namespace titan
