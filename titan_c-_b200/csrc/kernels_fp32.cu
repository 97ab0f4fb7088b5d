// FP32-flux translation unit: the Riemann solver's arithmetic in single
// precision. Reconstruction, the flux records (flux x area, FP64), the
// accumulation, update and CFL reduction stay in FP64, and faces that lie
// wholly in one side's wave region (supersonic faces) take their flux from the
// FP64 physical flux of that side (upwind_flux_fp64). Contraction to FMA is
// allowed here, and single-precision division and square root use the fast
// approximate forms (-prec-div=false, -prec-sqrt=false).
#include "face_dispatch.cuh"

namespace titan {

cudaError_t launch_face_flux_fp32(const FaceArgs& a, int nk, bool move, int variant, cudaStream_t s) {
    return face_flux_dispatch<float, false>(a, nk, move, variant, s);
}

cudaError_t launch_riemann_batch_fp32(long long n, const signed char* ns, const double* nrm, const double* w,
                                      const double* q1, const double* q2, double* flux, double* ds, int* rc,
                                      int flags, double gamma, cudaStream_t s) {
    riemann_batch_kernel<float><<<blocks_for(n, 128), 128, 0, s>>>(n, ns, nrm, w, q1, q2, flux, ds, rc, flags, gamma);
    return cudaGetLastError();
}

}  // namespace titan
