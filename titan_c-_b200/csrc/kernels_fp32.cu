// FP32-flux translation unit: the Riemann flux in single precision (the
// mixed-precision step keeps reconstruction, accumulation, update and the CFL
// reduction in FP64). Contraction to FMA is allowed here.
#include "launch.h"
#include "step_kernels.cuh"

namespace titan {

cudaError_t launch_face_flux_fp32(const FaceArgs& a, int nk, bool move, cudaStream_t s) {
    const unsigned int g = blocks_for(a.M.nface, kFaceBlock);
    if (nk == 0 && !move) face_flux_kernel<float, float, 0, false><<<g, kFaceBlock, 0, s>>>(a);
    else if (nk == 0 && move) face_flux_kernel<float, float, 0, true><<<g, kFaceBlock, 0, s>>>(a);
    else if (nk == 2 && !move) face_flux_kernel<float, float, 2, false><<<g, kFaceBlock, 0, s>>>(a);
    else if (nk == 2 && move) face_flux_kernel<float, float, 2, true><<<g, kFaceBlock, 0, s>>>(a);
    else return cudaErrorInvalidValue;
    return cudaGetLastError();
}

cudaError_t launch_riemann_batch_fp32(long long n, const signed char* ns, const double* nrm, const double* w,
                                      const double* q1, const double* q2, double* flux, double* ds, int* rc,
                                      int flags, double gamma, cudaStream_t s) {
    riemann_batch_kernel<float><<<blocks_for(n, 128), 128, 0, s>>>(n, ns, nrm, w, q1, q2, flux, ds, rc, flags, gamma);
    return cudaGetLastError();
}

}  // namespace titan
