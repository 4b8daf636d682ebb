/* bes_launch.h -- host entry points of the solver kernel variants
 * (one translation unit per units-per-lane class, so they build in parallel).
 *
 * Variant (U, RHS): U units per lane (1, 2, 4 for N <= 32, 64, 128);
 * RHS 0 keeps the operator in shared memory, RHS 1 keeps it in registers
 * (U = 1), RHS 2 is RHS 1 for launches whose systems all have 32 units,
 * RHS 3 stages one coupling matrix shared by the whole launch per CTA
 * (U = 2, 4). */
#ifndef BES_LAUNCH_H
#define BES_LAUNCH_H

#include <cuda_runtime.h>
#include <stddef.h>

#include "bes_device.h"

namespace bes {

/* shared-memory bytes one warp of class U needs (RHS 0-2) */
size_t warp_smem_bytes(int U);
/* dynamic shared memory of a CTA of `warps` warps of variant (U, RHS) */
size_t cta_smem_bytes(int U, int rhs, int warps);
/* most warps per CTA variant (U, RHS) allows */
int max_warps_per_block(int U, int rhs);
/* resident CTAs per SM for a CTA of `warps` warps of variant (U, RHS) */
cudaError_t occupancy(int U, int rhs, int warps, int* ctas_per_sm);
/* launch the persistent kernel of variant (U, RHS) */
cudaError_t launch(int U, int rhs, const DeviceProblem& P, int grid, int warps, cudaStream_t stream);

template <int U, int RHS>
size_t cta_smem_t(int warps);
template <int U, int RHS>
cudaError_t occupancy_t(int warps, int* ctas_per_sm);
template <int U, int RHS>
cudaError_t launch_t(const DeviceProblem& P, int grid, int warps, cudaStream_t stream);

}  // namespace bes

#endif
