/* bes_kernel_u1.cu -- solver kernel variants for systems of up to 32 units
 * (one unit per lane, one warp), the reference's BiCG recurrence. */
#include "bes_kernel_inst.cuh"

namespace bes {
BES_KERNEL_VARIANT(1, 1, 1, 0, BES_SMEM_WARP(1, 1))
BES_KERNEL_VARIANT(1, 2, 1, 0, BES_SMEM_WARP(1, 1))
BES_KERNEL_VARIANT(1, 5, 1, 0, BES_SMEM_WARP(1, 1))
BES_KERNEL_VARIANT(1, 6, 1, 0, BES_SMEM_WARP(1, 1))
BES_KERNEL_VARIANT(1, 7, 1, 0, BES_SMEM_BAND(1))
}  // namespace bes
