/* bes_kernel_u4.cu -- solver kernel variants for systems of up to 128 units (4 units per lane, one warp). */
#include "bes_kernel.cuh"
#include "bes_launch.h"

namespace bes {

template <>
size_t cta_smem_t<4, 0, 1>(int warps) { return (size_t)(warps / 1) * WarpSmem<4, 1>::BYTES; }

template <>
cudaError_t occupancy_t<4, 0, 1>(int warps, int* ctas_per_sm) {
    const size_t smem = cta_smem_t<4, 0, 1>(warps);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(bes_ensemble_kernel<4, 0, 1>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, bes_ensemble_kernel<4, 0, 1>, 32 * warps, smem);
}

template <>
cudaError_t launch_t<4, 0, 1>(const DeviceProblem& P, int grid, int warps, cudaStream_t stream) {
    bes_ensemble_kernel<4, 0, 1><<<grid, 32 * warps, cta_smem_t<4, 0, 1>(warps), stream>>>(P);
    return cudaGetLastError();
}

template <>
size_t cta_smem_t<4, 3, 1>(int warps) { return (size_t)SharedCSmem<4, 1>::C_BYTES + (size_t)(warps / 1) * SharedCSmem<4, 1>::WARP_BYTES; }

template <>
cudaError_t occupancy_t<4, 3, 1>(int warps, int* ctas_per_sm) {
    const size_t smem = cta_smem_t<4, 3, 1>(warps);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(bes_ensemble_kernel<4, 3, 1>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, bes_ensemble_kernel<4, 3, 1>, 32 * warps, smem);
}

template <>
cudaError_t launch_t<4, 3, 1>(const DeviceProblem& P, int grid, int warps, cudaStream_t stream) {
    bes_ensemble_kernel<4, 3, 1><<<grid, 32 * warps, cta_smem_t<4, 3, 1>(warps), stream>>>(P);
    return cudaGetLastError();
}

template <>
size_t cta_smem_t<4, 4, 1>(int warps) { return (size_t)SharedCSmem<4, 1>::C_BYTES + (size_t)(warps / 1) * SharedCSmem<4, 1>::WARP_BYTES; }

template <>
cudaError_t occupancy_t<4, 4, 1>(int warps, int* ctas_per_sm) {
    const size_t smem = cta_smem_t<4, 4, 1>(warps);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(bes_ensemble_kernel<4, 4, 1>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, bes_ensemble_kernel<4, 4, 1>, 32 * warps, smem);
}

template <>
cudaError_t launch_t<4, 4, 1>(const DeviceProblem& P, int grid, int warps, cudaStream_t stream) {
    bes_ensemble_kernel<4, 4, 1><<<grid, 32 * warps, cta_smem_t<4, 4, 1>(warps), stream>>>(P);
    return cudaGetLastError();
}

}  // namespace bes
