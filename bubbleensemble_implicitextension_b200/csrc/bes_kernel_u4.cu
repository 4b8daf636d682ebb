/* bes_kernel_u4.cu -- solver kernel variants for systems of up to 128 units
 * on one warp (four units per lane), the reference's BiCG recurrence. */
#include "bes_kernel_inst.cuh"

namespace bes {
BES_KERNEL_VARIANT(4, 0, 1, 0, BES_SMEM_WARP(4, 1))
BES_KERNEL_VARIANT(4, 3, 1, 0, BES_SMEM_SHARED(4, 1))
BES_KERNEL_VARIANT(4, 4, 1, 0, BES_SMEM_SHARED(4, 1))
}  // namespace bes
