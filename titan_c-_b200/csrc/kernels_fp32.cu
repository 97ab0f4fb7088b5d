// FP32-flux translation unit: the Riemann flux in single precision (the
// mixed-precision step keeps reconstruction, accumulation, update and the CFL
// reduction in FP64). Contraction to FMA is allowed here, and single-precision
// division and square root use the fast approximate forms (-prec-div=false,
// -prec-sqrt=false): the flux error budget is 1e-4, far above their few ulp.
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
