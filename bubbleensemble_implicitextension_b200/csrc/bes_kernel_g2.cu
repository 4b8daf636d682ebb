/* bes_kernel_g2.cu -- solver kernel variants for systems of up to 64 units (1 unit per lane, two warps). */
#include "bes_kernel.cuh"
#include "bes_launch.h"

namespace bes {

template <>
size_t cta_smem_t<1, 0, 2>(int warps) { return (size_t)(warps / 2) * WarpSmem<1, 2>::BYTES; }

template <>
cudaError_t occupancy_t<1, 0, 2>(int warps, int* ctas_per_sm) {
    const size_t smem = cta_smem_t<1, 0, 2>(warps);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(bes_ensemble_kernel<1, 0, 2>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, bes_ensemble_kernel<1, 0, 2>, 32 * warps, smem);
}

template <>
cudaError_t launch_t<1, 0, 2>(const DeviceProblem& P, int grid, int warps, cudaStream_t stream) {
    bes_ensemble_kernel<1, 0, 2><<<grid, 32 * warps, cta_smem_t<1, 0, 2>(warps), stream>>>(P);
    return cudaGetLastError();
}

template <>
size_t cta_smem_t<1, 3, 2>(int warps) { return (size_t)SharedCSmem<1, 2>::C_BYTES + (size_t)(warps / 2) * SharedCSmem<1, 2>::WARP_BYTES; }

template <>
cudaError_t occupancy_t<1, 3, 2>(int warps, int* ctas_per_sm) {
    const size_t smem = cta_smem_t<1, 3, 2>(warps);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(bes_ensemble_kernel<1, 3, 2>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, bes_ensemble_kernel<1, 3, 2>, 32 * warps, smem);
}

template <>
cudaError_t launch_t<1, 3, 2>(const DeviceProblem& P, int grid, int warps, cudaStream_t stream) {
    bes_ensemble_kernel<1, 3, 2><<<grid, 32 * warps, cta_smem_t<1, 3, 2>(warps), stream>>>(P);
    return cudaGetLastError();
}

template <>
size_t cta_smem_t<1, 4, 2>(int warps) { return (size_t)SharedCSmem<1, 2>::C_BYTES + (size_t)(warps / 2) * SharedCSmem<1, 2>::WARP_BYTES; }

template <>
cudaError_t occupancy_t<1, 4, 2>(int warps, int* ctas_per_sm) {
    const size_t smem = cta_smem_t<1, 4, 2>(warps);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(bes_ensemble_kernel<1, 4, 2>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, bes_ensemble_kernel<1, 4, 2>, 32 * warps, smem);
}

template <>
cudaError_t launch_t<1, 4, 2>(const DeviceProblem& P, int grid, int warps, cudaStream_t stream) {
    bes_ensemble_kernel<1, 4, 2><<<grid, 32 * warps, cta_smem_t<1, 4, 2>(warps), stream>>>(P);
    return cudaGetLastError();
}

}  // namespace bes
