/* bes_launch.cu -- dispatch from a run-time variant to the kernel instantiations. */
#include <algorithm>

#include "bes_kernel.cuh"
#include "bes_launch.h"

namespace bes {

namespace {

template <int U_, int RHS_, int G_, int REC_>
struct Tag {
    static constexpr int U = U_, RHS = RHS_, G = G_, REC = REC_;
};

template <int REC, class F>
bool dispatch_rec(Variant v, F&& f) {
    const int key = v.U * 100 + v.rhs * 10 + v.G;
    switch (key) {
        case 111: f(Tag<1, 1, 1, REC>{}); return true;
        case 121: f(Tag<1, 2, 1, REC>{}); return true;
        case 151: f(Tag<1, 5, 1, REC>{}); return true;
        case 161: f(Tag<1, 6, 1, REC>{}); return true;
        case 201: f(Tag<2, 0, 1, REC>{}); return true;
        case 231: f(Tag<2, 3, 1, REC>{}); return true;
        case 401: f(Tag<4, 0, 1, REC>{}); return true;
        case 431: f(Tag<4, 3, 1, REC>{}); return true;
        case 241: f(Tag<2, 4, 1, REC>{}); return true;
        case 441: f(Tag<4, 4, 1, REC>{}); return true;
        case 142: f(Tag<1, 4, 2, REC>{}); return true;
        case 144: f(Tag<1, 4, 4, REC>{}); return true;
        case 102: f(Tag<1, 0, 2, REC>{}); return true;
        case 132: f(Tag<1, 3, 2, REC>{}); return true;
        case 104: f(Tag<1, 0, 4, REC>{}); return true;
        case 134: f(Tag<1, 3, 4, REC>{}); return true;
        case 171: f(Tag<1, 7, 1, REC>{}); return true;
        case 172: f(Tag<1, 7, 2, REC>{}); return true;
        case 174: f(Tag<1, 7, 4, REC>{}); return true;
        default: return false;
    }
}

/* calls f(Tag<U, RHS, G, REC>{}) for the built variant v; false if v is not built */
template <class F>
bool dispatch(Variant v, F&& f) {
    if (v.rec == 0) return dispatch_rec<0>(v, f);
    if (v.rec == 1) return dispatch_rec<1>(v, f);
    return false;
}

}  // namespace

bool variant_exists(Variant v) {
    return dispatch(v, [](auto) {});
}

size_t cta_smem_bytes(Variant v, int warps) {
    size_t r = 0;
    dispatch(v, [&](auto t) { using T = decltype(t); r = cta_smem_t<T::U, T::RHS, T::G, T::REC>(warps, v.band); });
    return r;
}

int max_warps_per_block(Variant v) {
    /* the kernels' launch bounds: 256 threads with RHS 3 or G > 1, else 128 */
    const int cap = (v.rhs == 3 || v.rhs == 4 || v.rhs == 7 || v.G > 1) ? 8 : 4;
    int w = 0;
    while (w + v.G <= cap && cta_smem_bytes(v, w + v.G) <= 227 * 1024) w += v.G;
    return w;
}

cudaError_t occupancy(Variant v, int warps, int* ctas_per_sm) {
    cudaError_t e = cudaErrorInvalidValue;
    dispatch(v, [&](auto t) { using T = decltype(t); e = occupancy_t<T::U, T::RHS, T::G, T::REC>(warps, v.band, ctas_per_sm); });
    return e;
}

cudaError_t launch(Variant v, const DeviceProblem& P, int grid, int warps, cudaStream_t stream) {
    cudaError_t e = cudaErrorInvalidValue;
    dispatch(v, [&](auto t) { using T = decltype(t); e = launch_t<T::U, T::RHS, T::G, T::REC>(P, grid, warps, stream); });
    return e;
}

/* kernel variant of a units class: N <= 32 keeps the operator in registers
 * (rhs 2: every system has exactly 32 units); larger N runs one unit per lane
 * on 2 or 4 warps (or 2 or 4 units per lane on one warp) with W in shared
 * memory, or one staged copy of a matrix shared by the whole class when the
 * caller asked for shared coupling matrices (SharedCouplingMatrices).  With
 * banded coupling storage (band > 0) every class whose matrix is not staged
 * as a shared symmetric (N <= 32) or shared (N > 32) matrix runs the banded
 * operator, one unit per lane on 1, 2 or 4 warps. */
Variant class_variant(int cls, bool all32, bool shared, int warps_per_system, bool symmetric, int rec, int band) {
    if (cls == 0) {
        if (shared && symmetric) return Variant{1, all32 ? 6 : 5, 1, rec};   /* row of G in registers */
        if (band > 0) return Variant{1, 7, 1, rec, band};
        return Variant{1, all32 ? 2 : 1, 1, rec};
    }
    const int width = cls == 1 ? 2 : 4;
    if (!shared && band > 0) return Variant{1, 7, width, rec, band};   /* banded storage: one unit per lane */
    const int rhs = shared ? (symmetric ? 4 : 3) : 0;
    if (warps_per_system == 1) return Variant{width, rhs, 1, rec};
    return Variant{1, rhs, width, rec};
}

/* CTA shape of a launch of `count` systems: spread small ensembles over every
 * SM, fill SMs otherwise; `requested` > 0 asks for that many warps per CTA */
int class_warps_per_block(Variant v, int count, int sm_count, int requested) {
    const int cap = max_warps_per_block(v);
    int wpb = requested;
    if (wpb <= 0) {
        const int systems = count <= sm_count ? 1 : (count <= 2 * sm_count ? 2 : cap / v.G);
        wpb = systems * v.G;
    }
    wpb = std::max(v.G, std::min(wpb, cap)) / v.G * v.G;
    return wpb;
}

}  // namespace bes
