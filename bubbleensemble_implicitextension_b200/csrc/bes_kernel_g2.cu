/* bes_kernel_g2.cu -- solver kernel variants for systems of up to 64 units
 * (one unit per lane, two warps), the reference's BiCG recurrence. */
#include "bes_kernel_inst.cuh"

namespace bes {
BES_KERNEL_VARIANT(1, 0, 2, 0, BES_SMEM_WARP(1, 2))
BES_KERNEL_VARIANT(1, 3, 2, 0, BES_SMEM_SHARED(1, 2))
BES_KERNEL_VARIANT(1, 4, 2, 0, BES_SMEM_SHARED(1, 2))
BES_KERNEL_VARIANT(1, 7, 2, 0, BES_SMEM_BAND(2))
}  // namespace bes
