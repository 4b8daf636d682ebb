/* bes_kernel_u2_r1.cu -- solver kernel variants for systems of up to 64 units
 * on one warp (two units per lane), the single-reduction BiCG recurrence. */
#include "bes_kernel_inst.cuh"

namespace bes {
BES_KERNEL_VARIANT(2, 0, 1, 1, BES_SMEM_WARP(2, 1))
BES_KERNEL_VARIANT(2, 3, 1, 1, BES_SMEM_SHARED(2, 1))
BES_KERNEL_VARIANT(2, 4, 1, 1, BES_SMEM_SHARED(2, 1))
}  // namespace bes
