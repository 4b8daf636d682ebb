/* bes_launch.h -- host entry points of the solver kernel variants
 * (one translation unit per layout class, so they build in parallel).
 *
 * Variant (U, RHS, G): G warps per system with U units per lane (single warp:
 * U = 1, 2, 4 for N <= 32, 64, 128; multi-warp: U = 1 with G = 2, 4 for
 * N <= 64, 128).  RHS 0 keeps the operator in shared memory, RHS 1 keeps it
 * in registers (U = G = 1), RHS 2 is RHS 1 for launches whose systems all
 * have 32 units, RHS 3 stages one coupling matrix shared by the whole launch
 * per CTA (64 or 128 units), RHS 4 is RHS 3 for a symmetric shared matrix
 * (both BiCG products as row sums from one shared-memory read); RHS 5 / 6
 * (U = G = 1, N <= 32) keep a row of a shared symmetric matrix in registers
 * (6: every system has 32 units); RHS 7 (U = 1) keeps only the wrapping
 * band of banded coupling storage (CBW > 0).  Every variant exists with both BiCG
 * recurrences (REC 0: the reference's; 1: the single-reduction form). */
#ifndef BES_LAUNCH_H
#define BES_LAUNCH_H

#include <cuda_runtime.h>
#include <stddef.h>

#include "bes_device.h"

namespace bes {

/* a kernel variant; rec selects the BiCG recurrence (0: the reference's,
 * 1: the single-reduction form) */
struct Variant {
    int U, rhs, G;
    int rec = 0;
    int band = 0;   /* band width of the banded variant (RHS 7) */
};

/* is (U, RHS, G) one of the built variants */
bool variant_exists(Variant v);
/* dynamic shared memory of a CTA of `warps` warps (a multiple of G) */
size_t cta_smem_bytes(Variant v, int warps);
/* most warps per CTA the variant allows (a multiple of G; 0 if none fits) */
int max_warps_per_block(Variant v);
/* resident CTAs per SM for a CTA of `warps` warps */
cudaError_t occupancy(Variant v, int warps, int* ctas_per_sm);
/* launch the persistent kernel of the variant */
cudaError_t launch(Variant v, const DeviceProblem& P, int grid, int warps, cudaStream_t stream);

/* variant of units class cls (0: N <= 32, 1: N <= 64, 2: N <= 128); all32:
 * every system of the launch has 32 units; shared: the launch shares one
 * coupling matrix; warps_per_system 1 keeps every system on one warp; rec:
 * the BiCG recurrence */
Variant class_variant(int cls, bool all32, bool shared, int warps_per_system, bool symmetric = false, int rec = 0,
                      int band = 0);
/* warps per CTA for `count` systems of variant v (requested > 0: that many,
 * clamped to what the variant allows and rounded down to a multiple of G) */
int class_warps_per_block(Variant v, int count, int sm_count, int requested);

template <int U, int RHS, int G, int REC>
size_t cta_smem_t(int warps, int band);
template <int U, int RHS, int G, int REC>
cudaError_t occupancy_t(int warps, int band, int* ctas_per_sm);
template <int U, int RHS, int G, int REC>
cudaError_t launch_t(const DeviceProblem& P, int grid, int warps, cudaStream_t stream);

}  // namespace bes

#endif
