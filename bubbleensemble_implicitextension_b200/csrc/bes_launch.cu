/* bes_launch.cu -- dispatch from a run-time variant to the kernel instantiations. */
#include "bes_kernel.cuh"
#include "bes_launch.h"

namespace bes {

size_t warp_smem_bytes(int U) {
    switch (U) {
        case 1: return (size_t)WarpSmem<1>::BYTES;
        case 2: return (size_t)WarpSmem<2>::BYTES;
        default: return (size_t)WarpSmem<4>::BYTES;
    }
}

size_t cta_smem_bytes(int U, int rhs, int warps) {
    if (U == 1) return rhs == 2 ? cta_smem_t<1, 2>(warps) : cta_smem_t<1, 1>(warps);
    if (U == 2) return rhs == 3 ? cta_smem_t<2, 3>(warps) : cta_smem_t<2, 0>(warps);
    return rhs == 3 ? cta_smem_t<4, 3>(warps) : cta_smem_t<4, 0>(warps);
}

int max_warps_per_block(int U, int rhs) {
    const int cap = rhs == 3 ? 8 : 4;   /* the kernels' launch bounds: 256 and 128 threads */
    int w = 0;
    while (w < cap && cta_smem_bytes(U, rhs, w + 1) <= 227 * 1024) w++;
    return w;
}

cudaError_t occupancy(int U, int rhs, int warps, int* ctas_per_sm) {
    if (U == 1) return rhs == 2 ? occupancy_t<1, 2>(warps, ctas_per_sm) : occupancy_t<1, 1>(warps, ctas_per_sm);
    if (U == 2) return rhs == 3 ? occupancy_t<2, 3>(warps, ctas_per_sm) : occupancy_t<2, 0>(warps, ctas_per_sm);
    return rhs == 3 ? occupancy_t<4, 3>(warps, ctas_per_sm) : occupancy_t<4, 0>(warps, ctas_per_sm);
}

cudaError_t launch(int U, int rhs, const DeviceProblem& P, int grid, int warps, cudaStream_t stream) {
    if (U == 1) return rhs == 2 ? launch_t<1, 2>(P, grid, warps, stream) : launch_t<1, 1>(P, grid, warps, stream);
    if (U == 2) return rhs == 3 ? launch_t<2, 3>(P, grid, warps, stream) : launch_t<2, 0>(P, grid, warps, stream);
    return rhs == 3 ? launch_t<4, 3>(P, grid, warps, stream) : launch_t<4, 0>(P, grid, warps, stream);
}

}  // namespace bes
