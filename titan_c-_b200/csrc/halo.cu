// Halo exchange of a sharded step: whole-cell copies between the renumbered
// state and a flat device buffer that NCCL (or any copy) moves between ranks.
#include "halo.h"
#include "launch.h"

namespace titan {
namespace {

__global__ void halo_pack_kernel(const double* __restrict__ state, int ncell, const int* __restrict__ ids, int n,
                                 int ns, double* __restrict__ out) {
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q >= (long long)n * ns) return;
    const int i = (int)(q / ns), k = (int)(q % ns);
    out[q] = state[(size_t)k * ncell + ids[i]];
}

__global__ void halo_unpack_kernel(double* __restrict__ state, int ncell, const int* __restrict__ ids, int n, int ns,
                                   const double* __restrict__ in) {
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q >= (long long)n * ns) return;
    const int i = (int)(q / ns), k = (int)(q % ns);
    state[(size_t)k * ncell + ids[i]] = in[q];
}

}  // namespace

cudaError_t launch_halo_pack(const double* state, int ncell, const int* ids, int n, int ns, double* out,
                             cudaStream_t s) {
    if (n > 0) halo_pack_kernel<<<blocks_for((long long)n * ns, 256), 256, 0, s>>>(state, ncell, ids, n, ns, out);
    return cudaGetLastError();
}

cudaError_t launch_halo_unpack(double* state, int ncell, const int* ids, int n, int ns, const double* in,
                               cudaStream_t s) {
    if (n > 0) halo_unpack_kernel<<<blocks_for((long long)n * ns, 256), 256, 0, s>>>(state, ncell, ids, n, ns, in);
    return cudaGetLastError();
}

}  // namespace titan
