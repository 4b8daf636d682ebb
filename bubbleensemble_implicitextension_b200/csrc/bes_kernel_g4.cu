/* bes_kernel_g4.cu -- solver kernel variants for systems of up to 128 units (1 unit per lane, four warps). */
#include "bes_kernel.cuh"
#include "bes_launch.h"

namespace bes {

template <>
size_t cta_smem_t<1, 0, 4>(int warps) { return (size_t)(warps / 4) * WarpSmem<1, 4>::BYTES; }

template <>
cudaError_t occupancy_t<1, 0, 4>(int warps, int* ctas_per_sm) {
    const size_t smem = cta_smem_t<1, 0, 4>(warps);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(bes_ensemble_kernel<1, 0, 4>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, bes_ensemble_kernel<1, 0, 4>, 32 * warps, smem);
}

template <>
cudaError_t launch_t<1, 0, 4>(const DeviceProblem& P, int grid, int warps, cudaStream_t stream) {
    bes_ensemble_kernel<1, 0, 4><<<grid, 32 * warps, cta_smem_t<1, 0, 4>(warps), stream>>>(P);
    return cudaGetLastError();
}

template <>
size_t cta_smem_t<1, 3, 4>(int warps) { return (size_t)SharedCSmem<1, 4>::C_BYTES + (size_t)(warps / 4) * SharedCSmem<1, 4>::WARP_BYTES; }

template <>
cudaError_t occupancy_t<1, 3, 4>(int warps, int* ctas_per_sm) {
    const size_t smem = cta_smem_t<1, 3, 4>(warps);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(bes_ensemble_kernel<1, 3, 4>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, bes_ensemble_kernel<1, 3, 4>, 32 * warps, smem);
}

template <>
cudaError_t launch_t<1, 3, 4>(const DeviceProblem& P, int grid, int warps, cudaStream_t stream) {
    bes_ensemble_kernel<1, 3, 4><<<grid, 32 * warps, cta_smem_t<1, 3, 4>(warps), stream>>>(P);
    return cudaGetLastError();
}

template <>
size_t cta_smem_t<1, 4, 4>(int warps) { return (size_t)SharedCSmem<1, 4>::C_BYTES + (size_t)(warps / 4) * SharedCSmem<1, 4>::WARP_BYTES; }

template <>
cudaError_t occupancy_t<1, 4, 4>(int warps, int* ctas_per_sm) {
    const size_t smem = cta_smem_t<1, 4, 4>(warps);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(bes_ensemble_kernel<1, 4, 4>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, bes_ensemble_kernel<1, 4, 4>, 32 * warps, smem);
}

template <>
cudaError_t launch_t<1, 4, 4>(const DeviceProblem& P, int grid, int warps, cudaStream_t stream) {
    bes_ensemble_kernel<1, 4, 4><<<grid, 32 * warps, cta_smem_t<1, 4, 4>(warps), stream>>>(P);
    return cudaGetLastError();
}

}  // namespace bes
