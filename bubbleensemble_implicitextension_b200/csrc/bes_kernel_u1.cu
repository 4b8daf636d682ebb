/* bes_kernel_u1.cu -- solver kernel variants for systems of up to 32 units (1 unit per lane, one warp). */
#include "bes_kernel.cuh"
#include "bes_launch.h"

namespace bes {

template <>
size_t cta_smem_t<1, 1, 1>(int warps) { return (size_t)(warps / 1) * WarpSmem<1, 1>::BYTES; }

template <>
cudaError_t occupancy_t<1, 1, 1>(int warps, int* ctas_per_sm) {
    const size_t smem = cta_smem_t<1, 1, 1>(warps);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(bes_ensemble_kernel<1, 1, 1>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, bes_ensemble_kernel<1, 1, 1>, 32 * warps, smem);
}

template <>
cudaError_t launch_t<1, 1, 1>(const DeviceProblem& P, int grid, int warps, cudaStream_t stream) {
    bes_ensemble_kernel<1, 1, 1><<<grid, 32 * warps, cta_smem_t<1, 1, 1>(warps), stream>>>(P);
    return cudaGetLastError();
}

template <>
size_t cta_smem_t<1, 2, 1>(int warps) { return (size_t)(warps / 1) * WarpSmem<1, 1>::BYTES; }

template <>
cudaError_t occupancy_t<1, 2, 1>(int warps, int* ctas_per_sm) {
    const size_t smem = cta_smem_t<1, 2, 1>(warps);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(bes_ensemble_kernel<1, 2, 1>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, bes_ensemble_kernel<1, 2, 1>, 32 * warps, smem);
}

template <>
cudaError_t launch_t<1, 2, 1>(const DeviceProblem& P, int grid, int warps, cudaStream_t stream) {
    bes_ensemble_kernel<1, 2, 1><<<grid, 32 * warps, cta_smem_t<1, 2, 1>(warps), stream>>>(P);
    return cudaGetLastError();
}

template <>
size_t cta_smem_t<1, 5, 1>(int warps) { return (size_t)(warps / 1) * WarpSmem<1, 1>::BYTES; }

template <>
cudaError_t occupancy_t<1, 5, 1>(int warps, int* ctas_per_sm) {
    const size_t smem = cta_smem_t<1, 5, 1>(warps);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(bes_ensemble_kernel<1, 5, 1>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, bes_ensemble_kernel<1, 5, 1>, 32 * warps, smem);
}

template <>
cudaError_t launch_t<1, 5, 1>(const DeviceProblem& P, int grid, int warps, cudaStream_t stream) {
    bes_ensemble_kernel<1, 5, 1><<<grid, 32 * warps, cta_smem_t<1, 5, 1>(warps), stream>>>(P);
    return cudaGetLastError();
}

template <>
size_t cta_smem_t<1, 6, 1>(int warps) { return (size_t)(warps / 1) * WarpSmem<1, 1>::BYTES; }

template <>
cudaError_t occupancy_t<1, 6, 1>(int warps, int* ctas_per_sm) {
    const size_t smem = cta_smem_t<1, 6, 1>(warps);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(bes_ensemble_kernel<1, 6, 1>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, bes_ensemble_kernel<1, 6, 1>, 32 * warps, smem);
}

template <>
cudaError_t launch_t<1, 6, 1>(const DeviceProblem& P, int grid, int warps, cudaStream_t stream) {
    bes_ensemble_kernel<1, 6, 1><<<grid, 32 * warps, cta_smem_t<1, 6, 1>(warps), stream>>>(P);
    return cudaGetLastError();
}

}  // namespace bes
