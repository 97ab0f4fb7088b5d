// Second-order (TVD) faces with the FP32 Riemann flux (flags as
// kernels_fp32.cu). The reconstruction itself stays in FP64.
#include "face_dispatch.cuh"

namespace titan {

cudaError_t launch_face_flux_tvd_fp32(const FaceArgs& a, int nk, bool move, int variant, cudaStream_t s) {
    return face_flux_dispatch<float, true>(a, nk, move, variant, s);
}

}  // namespace titan
