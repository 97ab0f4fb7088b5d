// FP64 translation unit: geometry, FP64 face flux, cell update, permutations.
// Built with -fmad=false so that double-precision expressions round exactly as
// the reference's x86-64 build (no fused multiply-add contraction).
#include "face_dispatch.cuh"

namespace titan {

cudaError_t launch_move_nodes(const MeshView& M, const Params& P, const double* xyz1, double* xyz2,
                              const DevStatus* st, cudaStream_t s) {
    move_nodes_kernel<<<blocks_for(M.nnode, kGeomBlock), kGeomBlock, 0, s>>>(M, P, xyz1, xyz2, st);
    return cudaGetLastError();
}

cudaError_t launch_cell_geometry(const MeshView& M, const Layer& L, cudaStream_t s) {
    cell_geometry_kernel<<<blocks_for(M.ncell, kGeomBlock), kGeomBlock, 0, s>>>(M, L);
    return cudaGetLastError();
}

cudaError_t launch_face_geometry(const MeshView& M, const Layer& L, cudaStream_t s) {
    face_geometry_kernel<<<blocks_for(M.nface, kGeomBlock), kGeomBlock, 0, s>>>(M, L);
    return cudaGetLastError();
}

cudaError_t launch_face_flux_fp64(const FaceArgs& a, int nk, bool move, int variant, cudaStream_t s) {
    return face_flux_dispatch<double, false>(a, nk, move, variant, s);
}


static __global__ void godunov_batch_kernel(long long n, const double* __restrict__ nrm, const double* __restrict__ w,
                                            const double* __restrict__ q1, const double* __restrict__ q2,
                                            const signed char* __restrict__ contact, double gamma,
                                            double* __restrict__ flux, double* __restrict__ ds, int* __restrict__ rc) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    double out[5] = {0, 0, 0, 0, 0}, d[3] = {0, 0, 0};
    rc[i] = godunov_exact(nrm + 3 * i, w[i], q1 + 5 * i, q2 + 5 * i, contact[i], gamma, out, d);
    for (int k = 0; k < 5; ++k) flux[5 * i + k] = out[k];
    for (int k = 0; k < 3; ++k) ds[3 * i + k] = d[k];
}

cudaError_t launch_godunov_batch(long long n, const double* nrm, const double* w, const double* q1, const double* q2,
                                 const signed char* contact, double gamma, double* flux, double* ds, int* rc,
                                 cudaStream_t s) {
    godunov_batch_kernel<<<blocks_for(n, 128), 128, 0, s>>>(n, nrm, w, q1, q2, contact, gamma, flux, ds, rc);
    return cudaGetLastError();
}

cudaError_t launch_gather(const double* src, double* dst, const int* perm, int n, int nfields, cudaStream_t s) {
    gather_fields_kernel<<<blocks_for(n, 256), 256, 0, s>>>(src, dst, perm, n, nfields);
    return cudaGetLastError();
}

cudaError_t launch_scatter(const double* src, double* dst, const int* perm, int n, int nfields, cudaStream_t s) {
    scatter_fields_kernel<<<blocks_for(n, 256), 256, 0, s>>>(src, dst, perm, n, nfields);
    return cudaGetLastError();
}

cudaError_t launch_riemann_batch_fp64(long long n, const signed char* ns, const double* nrm, const double* w,
                                      const double* q1, const double* q2, double* flux, double* ds, int* rc,
                                      int flags, double gamma, cudaStream_t s) {
    riemann_batch_kernel<double><<<blocks_for(n, 128), 128, 0, s>>>(n, ns, nrm, w, q1, q2, flux, ds, rc, flags, gamma);
    return cudaGetLastError();
}

}  // namespace titan
