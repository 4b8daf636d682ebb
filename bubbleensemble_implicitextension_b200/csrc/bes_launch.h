/* bes_launch.h -- host entry points of the per-class solver kernels
 * (one translation unit per units-per-lane class, so they build in parallel). */
#ifndef BES_LAUNCH_H
#define BES_LAUNCH_H

#include <cuda_runtime.h>
#include <stddef.h>

#include "bes_device.h"

namespace bes {

/* shared-memory bytes one warp of class U needs */
size_t warp_smem_bytes(int U);
/* resident CTAs per SM for a CTA of `warps` warps of class U */
cudaError_t occupancy(int U, int warps, int* ctas_per_sm);
/* launch the persistent kernel of class U */
cudaError_t launch(int U, const DeviceProblem& P, int grid, int warps, cudaStream_t stream);

template <int U>
size_t warp_smem_bytes_t();
template <int U>
cudaError_t occupancy_t(int warps, int* ctas_per_sm);
template <int U>
cudaError_t launch_t(const DeviceProblem& P, int grid, int warps, cudaStream_t stream);

}  // namespace bes

#endif
