/* bes_kernel_g2_r1.cu -- solver kernel variants for systems of up to 64 units
 * (one unit per lane, two warps), the single-reduction BiCG recurrence. */
#include "bes_kernel_inst.cuh"

namespace bes {
BES_KERNEL_VARIANT(1, 0, 2, 1, BES_SMEM_WARP(1, 2))
BES_KERNEL_VARIANT(1, 3, 2, 1, BES_SMEM_SHARED(1, 2))
BES_KERNEL_VARIANT(1, 4, 2, 1, BES_SMEM_SHARED(1, 2))
BES_KERNEL_VARIANT(1, 7, 2, 1, BES_SMEM_BAND(2))
}  // namespace bes
