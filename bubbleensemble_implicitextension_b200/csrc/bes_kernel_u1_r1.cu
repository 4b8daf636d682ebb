/* bes_kernel_u1_r1.cu -- solver kernel variants for systems of up to 32 units
 * (one unit per lane, one warp), the single-reduction BiCG recurrence. */
#include "bes_kernel_inst.cuh"

namespace bes {
BES_KERNEL_VARIANT(1, 1, 1, 1, BES_SMEM_WARP(1, 1))
BES_KERNEL_VARIANT(1, 2, 1, 1, BES_SMEM_WARP(1, 1))
BES_KERNEL_VARIANT(1, 5, 1, 1, BES_SMEM_WARP(1, 1))
BES_KERNEL_VARIANT(1, 6, 1, 1, BES_SMEM_WARP(1, 1))
BES_KERNEL_VARIANT(1, 7, 1, 1, BES_SMEM_BAND(1))
}  // namespace bes
