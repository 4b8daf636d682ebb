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

cudaError_t occupancy(int U, int rhs, int warps, int* ctas_per_sm) {
    if (U == 1) return rhs == 2 ? occupancy_t<1, 2>(warps, ctas_per_sm) : occupancy_t<1, 1>(warps, ctas_per_sm);
    if (U == 2) return occupancy_t<2, 0>(warps, ctas_per_sm);
    return occupancy_t<4, 0>(warps, ctas_per_sm);
}

cudaError_t launch(int U, int rhs, const DeviceProblem& P, int grid, int warps, cudaStream_t stream) {
    if (U == 1) return rhs == 2 ? launch_t<1, 2>(P, grid, warps, stream) : launch_t<1, 1>(P, grid, warps, stream);
    if (U == 2) return launch_t<2, 0>(P, grid, warps, stream);
    return launch_t<4, 0>(P, grid, warps, stream);
}

}  // namespace bes
