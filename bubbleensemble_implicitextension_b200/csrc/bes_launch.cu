/* bes_launch.cu -- dispatch from a run-time class to the per-class kernels. */
#include "bes_launch.h"

namespace bes {

size_t warp_smem_bytes(int U) {
    switch (U) {
        case 1: return warp_smem_bytes_t<1>();
        case 2: return warp_smem_bytes_t<2>();
        default: return warp_smem_bytes_t<4>();
    }
}

cudaError_t occupancy(int U, int warps, int* ctas_per_sm) {
    switch (U) {
        case 1: return occupancy_t<1>(warps, ctas_per_sm);
        case 2: return occupancy_t<2>(warps, ctas_per_sm);
        default: return occupancy_t<4>(warps, ctas_per_sm);
    }
}

cudaError_t launch(int U, const DeviceProblem& P, int grid, int warps, cudaStream_t stream) {
    switch (U) {
        case 1: return launch_t<1>(P, grid, warps, stream);
        case 2: return launch_t<2>(P, grid, warps, stream);
        default: return launch_t<4>(P, grid, warps, stream);
    }
}

}  // namespace bes
