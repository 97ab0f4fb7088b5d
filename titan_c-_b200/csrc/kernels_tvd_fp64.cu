// Second-order (TVD) faces, FP64 translation unit (-fmad=false, like
// kernels_fp64.cu): the face-flux kernel with the second-order reconstruction
// of Setka_gran_snos.cpp:188-735, and the neighbour search of Setka::Init_TVD.
#include "face_dispatch.cuh"

namespace titan {

cudaError_t launch_face_flux_tvd_fp64(const FaceArgs& a, int nk, bool move, int variant, cudaStream_t s) {
    return face_flux_dispatch<double, true>(a, nk, move, variant, s);
}

cudaError_t launch_tvd_neighbours(const MeshView& M, const Layer& L, int* aa, int* bb, cudaStream_t s) {
    tvd_neighbours_kernel<<<blocks_for(M.nface, kGeomBlock), kGeomBlock, 0, s>>>(M, L, aa, bb);
    return cudaGetLastError();
}

}  // namespace titan
