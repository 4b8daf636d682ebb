/* bes_kernel_inst.cuh -- host entry points (shared-memory size, occupancy,
 * launch) of one solver kernel instantiation; each bes_kernel_*.cu unit
 * instantiates the variants of one layout class with one BiCG recurrence, so
 * the units compile in parallel. */
#ifndef BES_KERNEL_INST_CUH
#define BES_KERNEL_INST_CUH

#include "bes_kernel.cuh"
#include "bes_launch.h"

/* SMEM: dynamic shared memory of a CTA of `warps` warps (`band`: the band width of the banded variant) */
#define BES_KERNEL_VARIANT(U_, RHS_, G_, REC_, SMEM)                                                          \
    template <>                                                                                               \
    size_t cta_smem_t<U_, RHS_, G_, REC_>(int warps, int band) {                                              \
        (void)band;                                                                                           \
        return (SMEM);                                                                                        \
    }                                                                                                         \
    template <>                                                                                               \
    cudaError_t occupancy_t<U_, RHS_, G_, REC_>(int warps, int band, int* ctas_per_sm) {                      \
        const size_t smem = cta_smem_t<U_, RHS_, G_, REC_>(warps, band);                                      \
        if (smem > 48 * 1024) {                                                                               \
            cudaError_t e = cudaFuncSetAttribute(bes_ensemble_kernel<U_, RHS_, G_, REC_>,                     \
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);     \
            if (e != cudaSuccess) return e;                                                                   \
        }                                                                                                     \
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, bes_ensemble_kernel<U_, RHS_, G_, REC_>, \
                                                             32 * warps, smem);                               \
    }                                                                                                         \
    template <>                                                                                               \
    cudaError_t launch_t<U_, RHS_, G_, REC_>(const DeviceProblem& P, int grid, int warps, cudaStream_t stream) { \
        bes_ensemble_kernel<U_, RHS_, G_, REC_><<<grid, 32 * warps, cta_smem_t<U_, RHS_, G_, REC_>(warps, P.band_width), \
                                                  stream>>>(P);                                               \
        return cudaGetLastError();                                                                            \
    }

/* per-system shared memory (operator or staged matrix per system) */
#define BES_SMEM_WARP(U_, G_) (size_t)(warps / (G_)) * WarpSmem<U_, G_>::BYTES
/* per-system band of the coupling matrix, sized by the run-time band width */
#define BES_SMEM_BAND(G_) (size_t)(warps / (G_)) * (size_t)BandSmem<G_>::doubles(band) * 8
/* one staged matrix per CTA plus per-system vectors */
#define BES_SMEM_SHARED(U_, G_) \
    (size_t)SharedCSmem<U_, G_>::C_BYTES + (size_t)(warps / (G_)) * SharedCSmem<U_, G_>::WARP_BYTES

#endif
