/* bes_kernel_u2.cu -- solver kernel variants for systems of up to 64 units
 * (2 unit(s) per lane). */
#include "bes_kernel.cuh"
#include "bes_launch.h"

namespace bes {

template <>
size_t cta_smem_t<2, 0>(int warps) { return (size_t)warps * WarpSmem<2>::BYTES; }

template <>
cudaError_t occupancy_t<2, 0>(int warps, int* ctas_per_sm) {
    const size_t smem = cta_smem_t<2, 0>(warps);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(bes_ensemble_kernel<2, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
    }
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, bes_ensemble_kernel<2, 0>, 32 * warps, smem);
}

template <>
cudaError_t launch_t<2, 0>(const DeviceProblem& P, int grid, int warps, cudaStream_t stream) {
    bes_ensemble_kernel<2, 0><<<grid, 32 * warps, cta_smem_t<2, 0>(warps), stream>>>(P);
    return cudaGetLastError();
}
template <>
size_t cta_smem_t<2, 3>(int warps) { return (size_t)SharedCSmem<2>::C_BYTES + (size_t)warps * SharedCSmem<2>::WARP_BYTES; }

template <>
cudaError_t occupancy_t<2, 3>(int warps, int* ctas_per_sm) {
    const size_t smem = cta_smem_t<2, 3>(warps);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(bes_ensemble_kernel<2, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
    }
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, bes_ensemble_kernel<2, 3>, 32 * warps, smem);
}

template <>
cudaError_t launch_t<2, 3>(const DeviceProblem& P, int grid, int warps, cudaStream_t stream) {
    bes_ensemble_kernel<2, 3><<<grid, 32 * warps, cta_smem_t<2, 3>(warps), stream>>>(P);
    return cudaGetLastError();
}
}  // namespace bes
