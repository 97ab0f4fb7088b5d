// Halo exchange of a sharded step (halo.cu): copies between a context's
// renumbered cell state and a caller's device buffer of whole cells.
#pragma once
#include <cuda_runtime.h>

namespace titan {

// out[i][k] = state[k][ids[i]] for i < n, k < ns (cells packed whole, so one
// peer's cells are one contiguous slice of the buffer).
cudaError_t launch_halo_pack(const double* state, int ncell, const int* ids, int n, int ns, double* out,
                             cudaStream_t s);
// state[k][ids[i]] = in[i][k].
cudaError_t launch_halo_unpack(double* state, int ncell, const int* ids, int n, int ns, const double* in,
                               cudaStream_t s);

}  // namespace titan
