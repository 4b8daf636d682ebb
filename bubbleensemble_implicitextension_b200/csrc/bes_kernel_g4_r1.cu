/* bes_kernel_g4_r1.cu -- solver kernel variants for systems of up to 128 units
 * (one unit per lane, four warps), the single-reduction BiCG recurrence. */
#include "bes_kernel_inst.cuh"

namespace bes {
BES_KERNEL_VARIANT(1, 0, 4, 1, BES_SMEM_WARP(1, 4))
BES_KERNEL_VARIANT(1, 3, 4, 1, BES_SMEM_SHARED(1, 4))
BES_KERNEL_VARIANT(1, 4, 4, 1, BES_SMEM_SHARED(1, 4))
BES_KERNEL_VARIANT(1, 7, 4, 1, BES_SMEM_BAND(4))
}  // namespace bes
