/*
 * bes_noalloc.cu -- the ensemble solve for callers that cannot allocate
 * device memory.
 *
 * Who needs it: a host application that owns all of the GPU's memory itself
 * (a framework that reserves the device up front and hands out slices from
 * its own pool, or a real-time loop in which a cudaMalloc could block or
 * synchronise the device) can lay out every input and output array of an
 * ensemble in memory it already holds, but it cannot let a library call
 * cudaMalloc.  bes_create() allocates; bes_solve_periods_noalloc() does not.
 *
 * The solver kernel needs scratch memory besides the caller's arrays: one
 * work counter per units-per-lane class and the order in which warps pick up
 * systems.  Here that scratch is the file-scope device array g_scratch
 * below, of a fixed size: BES_NOALLOC_MAX_SYSTEMS systems.  Every GPU that
 * loads the library holds it (256 KiB + 16 B) until the process exits.
 *
 * Host code cannot use g_scratch's name as a device address, so on the first
 * call on a device (with that device current) the entry point asks the
 * runtime for the address with cudaGetSymbolAddress and keeps it; later calls
 * on that device reuse it.  That first call should therefore come before any
 * stream capture.  Each call re-zeroes the counters and rewrites the order
 * before its launches; all calls share the one array, so calls whose work
 * overlaps on the GPU (e.g. on two streams at once) race on it and must be
 * serialised by the caller.
 */
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "../../include/bes.h"
#include "bes_launch.h"
#include "bes_status.h"
#ifndef BES_SYSTEM_DEFINITION
#include "km_model.cuh"
#else
#include BES_SYSTEM_DEFINITION
#endif

#define BES_NOALLOC_MAX_DEVICES 64

namespace {

/* [0..3]: work counters of the three classes; [4..]: processing order */
static __device__ __align__(256) int32_t g_scratch[4 + BES_NOALLOC_MAX_SYSTEMS];

int32_t* g_scratch_addr[BES_NOALLOC_MAX_DEVICES] = {};
std::once_flag g_scratch_once[BES_NOALLOC_MAX_DEVICES];
cudaError_t g_scratch_err[BES_NOALLOC_MAX_DEVICES] = {};

int units_class(int n) { return n <= 32 ? 0 : (n <= 64 ? 1 : 2); }

/* Zero the counters and write each class's systems, in index order, into its
 * segment of the order: warp c handles class c, 32 systems per ballot.  The
 * order is first filled with -1, which the solver kernel skips: if the device
 * unit counts disagree with the host copy the plan was made from, a class
 * segment may be left partly unwritten, and no stale index from an earlier
 * call survives in it. */
__global__ void noalloc_prepare(const int32_t* __restrict__ units, int n, int32_t* scratch, int begin0, int begin1,
                                int begin2) {
    const int lane = threadIdx.x & 31, cls = threadIdx.x >> 5;
    if (threadIdx.x < 4) scratch[threadIdx.x] = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) scratch[4 + i] = -1;
    __syncthreads();
    if (cls > 2) return;
    int pos = 4 + (cls == 0 ? begin0 : (cls == 1 ? begin1 : begin2));
    for (int base = 0; base < n; base += 32) {
        const int s = base + lane;
        const int u = s < n ? units[s] : 0;
        const bool mine = s < n && (u <= 32 ? 0 : (u <= 64 ? 1 : 2)) == cls;
        const unsigned m = __ballot_sync(0xffffffffu, mine);
        const int at = pos + __popc(m & ((1u << lane) - 1u));
        if (mine && at < 4 + n) scratch[at] = s; /* stays inside the order even if units disagree with units_host */
        pos += __popc(m);
    }
}

bes_status report(const bes_noalloc_problem* p, bes_status st, const char* fmt, long long a, long long b) {
    if (p && p->error_message && p->error_capacity > 0)
        std::snprintf(p->error_message, (size_t)p->error_capacity, fmt, a, b);
    return st;
}

}  // namespace

extern "C" bes_status bes_solve_periods_noalloc(const bes_noalloc_problem* p, int32_t n_periods, int32_t reset_at,
                                                void* stream) {
    if (!p) return BES_ERR_ARGUMENT;
    if (p->n_systems < 0 || p->n_systems > BES_NOALLOC_MAX_SYSTEMS)
        return report(p, BES_ERR_ARGUMENT,
                      "bes_solve_periods_noalloc: %lld systems requested; the no-allocation scratch holds at most %lld",
                      (long long)p->n_systems, (long long)BES_NOALLOC_MAX_SYSTEMS);
    if (n_periods < 0) return report(p, BES_ERR_ARGUMENT, "bes_solve_periods_noalloc: n_periods %lld < %lld", (long long)n_periods, 0LL);
    if (p->n_systems == 0) return BES_OK;
    if (!p->units_host || !p->units || !p->unit_offset || !p->coupling_offset || !p->coupling || !p->state ||
        !p->upar || !p->time_domain || !p->actual_time || !p->rtol || !p->atol || !p->event_tol || !p->event_dir ||
        !p->n_accepted || !p->n_rejected || !p->n_bicg_iter || !p->n_rhs || !p->status ||
        (BES_MODEL_NUA > 0 && (!p->uacc || !p->uacc_reset)) || (BES_MODEL_NIUA > 0 && (!p->iuacc || !p->iuacc_reset)) ||
        (BES_MODEL_NSP > 0 && !p->spar) || (BES_MODEL_NSA > 0 && !p->sacc) || (BES_MODEL_NISA > 0 && !p->isacc) ||
        (BES_MODEL_NGP > 0 && !p->gpar) || (BES_MODEL_NIGP > 0 && !p->igpar) ||
        (p->ndo > 0 && (!p->dense_time || !p->dense_state || !p->dense_index)))
        return report(p, BES_ERR_ARGUMENT, "bes_solve_periods_noalloc: a required array pointer is null", 0, 0);
    if (p->algorithm != BES_RK4 && p->algorithm != BES_RKCK45)
        return report(p, BES_ERR_ARGUMENT, "bes_solve_periods_noalloc: unknown algorithm %lld", (long long)p->algorithm, 0);
    if (p->bicg_recurrence != 0 && p->bicg_recurrence != 1)
        return report(p, BES_ERR_ARGUMENT, "bes_solve_periods_noalloc: bicg_recurrence %lld is not 0 or 1",
                      (long long)p->bicg_recurrence, 0);

    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= BES_NOALLOC_MAX_DEVICES)
        return report(p, BES_ERR_CUDA, "bes_solve_periods_noalloc: no usable current device (%lld)", (long long)dev, 0);
    /* once per device, with that device current: the device address of g_scratch */
    std::call_once(g_scratch_once[dev], [dev]() {
        g_scratch_err[dev] = cudaGetSymbolAddress((void**)&g_scratch_addr[dev], g_scratch);
    });
    if (g_scratch_err[dev] != cudaSuccess || !g_scratch_addr[dev])
        return report(p, BES_ERR_CUDA, "bes_solve_periods_noalloc: cudaGetSymbolAddress failed on device %lld (cudaError %lld)",
                      (long long)dev, (long long)g_scratch_err[dev]);
    int32_t* scratch = g_scratch_addr[dev];

    /* launch plan from the host copy of the unit counts (no host allocation either) */
    int count[3] = {0, 0, 0};
    bool all32 = true;
    for (int s = 0; s < p->n_systems; s++) {
        const int n = p->units_host[s];
        if (n < 1 || n > 128)
            return report(p, BES_ERR_ARGUMENT, "bes_solve_periods_noalloc: system %lld has %lld units (1..128)", (long long)s,
                          (long long)n);
        count[units_class(n)]++;
        if (units_class(n) == 0 && n != 32) all32 = false;
    }
    const int begin[3] = {0, count[0], count[0] + count[1]};
    /* options: 0 takes the SolverOption default (Interface.cuh:613-618), a negative value is an error */
    const double opt[5] = {p->dt0, p->dtmin, p->dtmax, p->grow, p->shrink};
    const double dflt[5] = {1e-2, 1e-12, 1e6, 5.0, 0.1};
    const char* opt_name[5] = {"dt0", "dtmin", "dtmax", "grow", "shrink"};
    double val[5];
    for (int k = 0; k < 5; k++) {
        if (!(opt[k] >= 0.0)) {
            if (p->error_message && p->error_capacity > 0)
                std::snprintf(p->error_message, (size_t)p->error_capacity,
                              "bes_solve_periods_noalloc: option %s = %g is negative or not a number", opt_name[k], opt[k]);
            return BES_ERR_ARGUMENT;
        }
        val[k] = opt[k] == 0.0 ? dflt[k] : opt[k];
    }
    /* the launch shapes, checked before anything is queued */
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1) sms = 148;
    bes::Variant var[3];
    int wpb[3] = {0, 0, 0}, grid[3] = {0, 0, 0};
    cudaError_t e = cudaSuccess;
    for (int cls = 0; cls < 3; cls++) {
        if (count[cls] == 0) continue;
        var[cls] = bes::class_variant(cls, all32, false, 0, false, p->bicg_recurrence);
        const bes::Variant& v = var[cls];
        if (bes::max_warps_per_block(v) < v.G)
            return report(p, BES_ERR_CUDA, "bes_solve_periods_noalloc: kernel class %lld (%lld warps per system) does not fit in shared memory",
                          (long long)cls, (long long)v.G);
        wpb[cls] = bes::class_warps_per_block(v, count[cls], sms, p->warps_per_block);
        int per_sm = 0;
        e = bes::occupancy(v, wpb[cls], &per_sm);
        if (e != cudaSuccess || per_sm < 1)
            return report(p, BES_ERR_CUDA, "bes_solve_periods_noalloc: kernel class %lld cannot be resident (cudaError %lld)",
                          (long long)cls, (long long)e);
        const int needed = (count[cls] + wpb[cls] / v.G - 1) / (wpb[cls] / v.G);
        grid[cls] = needed < per_sm * sms ? needed : per_sm * sms;
    }
    cudaStream_t st = (cudaStream_t)stream;
    /* an error left pending by the caller's earlier work is reported as such (and not cleared) */
    e = cudaPeekAtLastError();
    if (e != cudaSuccess)
        return report(p, BES_ERR_CUDA, "bes_solve_periods_noalloc: a CUDA error from earlier work is pending (cudaError %lld)",
                      (long long)e, 0);
    noalloc_prepare<<<1, 96, 0, st>>>(p->units, p->n_systems, scratch, begin[0], begin[1], begin[2]);
    e = cudaGetLastError();
    if (e != cudaSuccess)
        return report(p, BES_ERR_CUDA, "bes_solve_periods_noalloc: prepare launch failed (cudaError %lld)", (long long)e, 0);

    bes::DeviceProblem P = {};
    P.n_systems = p->n_systems;
    P.total_units = p->total_units;
    P.units = p->units;
    P.unit_offset = p->unit_offset;
    P.coupling_offset = p->coupling_offset;
    P.coupling = p->coupling;
    P.state = p->state;
    P.upar = p->upar;
    P.uacc = p->uacc;
    P.iuacc = p->iuacc;
    P.spar = p->spar;
    P.sacc = p->sacc;
    P.isacc = p->isacc;
    P.gpar = p->gpar;
    P.igpar = p->igpar;
    P.time_domain = p->time_domain;
    P.actual_time = p->actual_time;
    P.rtol = p->rtol;
    P.atol = p->atol;
    P.event_tol = p->event_tol;
    P.event_dir = p->event_dir;
    P.dt0 = val[0];
    P.dtmin = val[1];
    P.dtmax = val[2];
    P.grow = val[3];
    P.shrink = val[4];
    P.algorithm = p->algorithm;
    P.bicg_max_iter = p->bicg_max_iter > 0 ? p->bicg_max_iter : 19;
    P.max_steps_per_period = p->max_steps_per_period > 0 ? p->max_steps_per_period : 1000000;
    P.ndo = p->ndo;
    P.do_save_frequency = p->do_save_frequency > 0 ? p->do_save_frequency : 1;
    P.do_min_dt = p->do_min_dt;
    P.dense_time = p->dense_time;
    P.dense_state = p->dense_state;
    P.dense_index = p->dense_index;
    P.n_accepted = (unsigned long long*)p->n_accepted;
    P.n_rejected = (unsigned long long*)p->n_rejected;
    P.n_bicg_iter = (unsigned long long*)p->n_bicg_iter;
    P.n_rhs = (unsigned long long*)p->n_rhs;
    P.status = p->status;
    P.n_periods = n_periods;
    P.reset_at = reset_at;
    P.uacc_reset = p->uacc_reset;
    P.iuacc_reset = p->iuacc_reset;

    for (int cls = 0; cls < 3; cls++) {
        if (count[cls] == 0) continue;
        P.order = scratch + 4 + begin[cls];
        P.n_active = count[cls];
        P.work_counter = scratch + cls;
        e = bes::launch(var[cls], P, grid[cls], wpb[cls], st);
        if (e != cudaSuccess)
            return report(p, BES_ERR_CUDA, "bes_solve_periods_noalloc: launch of class %lld failed (cudaError %lld)",
                          (long long)cls, (long long)e);
    }
    return BES_OK;
}
