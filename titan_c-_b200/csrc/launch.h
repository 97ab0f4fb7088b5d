// Host-callable launchers of the step kernels (implemented in kernels_fp64.cu
// and kernels_tvd_fp64.cu, built with -fmad=false, and kernels_fp32.cu and
// kernels_tvd_fp32.cu, built with contraction on).
#pragma once
#include <cuda_runtime.h>

#include "step_types.h"

namespace titan {

constexpr int kGeomBlock = 256;

// Launch shapes the autotuner chooses from: threads per block and the minimum
// resident blocks per SM requested from the register allocator.
struct FaceVariant {
    int block, min_blocks;
};
constexpr int kFaceVariants = 7;
constexpr FaceVariant kFaceVariant[kFaceVariants] = {{128, 1}, {128, 3}, {128, 4}, {256, 2}, {64, 8}, {128, 5},
                                                     {128, 6}};
// overflow > 0: the staged update (face records in shared memory, a bulk copy
// per block plus `overflow` cp.async slots per thread); needs the faces sorted
// by cells[0] (CellArgs::owner_start)
struct CellVariant {
    int block, min_blocks, overflow;
};
constexpr int kCellVariants = 9;
constexpr CellVariant kCellVariant[kCellVariants] = {{256, 1, 0}, {128, 1, 0}, {512, 1, 0}, {256, 4, 0}, {128, 8, 0},
                                                     {256, 3, 0}, {128, 3, 3}, {64, 6, 3},  {128, 4, 1}};

cudaError_t launch_move_nodes(const MeshView& M, const Params& P, const double* xyz1, double* xyz2,
                              const DevStatus* st, cudaStream_t s);
cudaError_t launch_cell_geometry(const MeshView& M, const Layer& L, cudaStream_t s);
cudaError_t launch_face_geometry(const MeshView& M, const Layer& L, cudaStream_t s);
cudaError_t launch_face_flux_fp64(const FaceArgs& a, int nk, bool move, int variant, cudaStream_t s);
cudaError_t launch_face_flux_fp32(const FaceArgs& a, int nk, bool move, int variant, cudaStream_t s);
// second-order faces (kernels_tvd_fp64.cu, kernels_tvd_fp32.cu)
cudaError_t launch_face_flux_tvd_fp64(const FaceArgs& a, int nk, bool move, int variant, cudaStream_t s);
cudaError_t launch_face_flux_tvd_fp32(const FaceArgs& a, int nk, bool move, int variant, cudaStream_t s);
cudaError_t launch_tvd_neighbours(const MeshView& M, const Layer& L, int* aa, int* bb, cudaStream_t s);
// the flux buffer holds FP64 records in every mode
cudaError_t launch_cell_update(const CellArgs& a, int nk, bool move, int src, int variant, cudaStream_t s);
// once per process, before any launch (sets the staged kernels' shared-memory size)
cudaError_t cell_update_prepare();
cudaError_t launch_gather(const double* src, double* dst, const int* perm, int n, int nfields, cudaStream_t s);
cudaError_t launch_scatter(const double* src, double* dst, const int* perm, int n, int nfields, cudaStream_t s);
cudaError_t launch_riemann_batch_fp64(long long n, const signed char* ns, const double* nrm, const double* w,
                                      const double* q1, const double* q2, double* flux, double* ds, int* rc,
                                      int flags, double gamma, cudaStream_t s);
cudaError_t launch_riemann_batch_fp32(long long n, const signed char* ns, const double* nrm, const double* w,
                                      const double* q1, const double* q2, double* flux, double* ds, int* rc,
                                      int flags, double gamma, cudaStream_t s);

cudaError_t launch_godunov_batch(long long n, const double* nrm, const double* w, const double* q1, const double* q2,
                                 const signed char* contact, double gamma, double* flux, double* ds, int* rc,
                                 cudaStream_t s);

inline unsigned int blocks_for(long long n, int bs) { return (unsigned int)((n + bs - 1) / bs); }

}  // namespace titan
