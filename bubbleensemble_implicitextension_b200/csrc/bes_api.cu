/*
 * bes_api.cu -- host side of the C ABI declared in include/bes.h.
 *
 * It owns what the reference's ProblemSolver owns
 * (SourceCodes/CoupledSystems_PerBlock_Interface.cuh:135-248, :354-714):
 * pinned host mirrors and device arrays of every variable, the solver
 * options, one CUDA stream and a synchronisation event.  Instead of exit()
 * every error returns a bes_status and leaves a message in the handle.
 *
 * Launch plan of bes_solve_periods: systems are grouped by units-per-lane
 * class (U = 1, 2, 4 for N <= 32, 64, 128), ordered costliest first inside a
 * class, and each non-empty class gets one launch of the persistent kernel
 * (a work counter per class hands systems to warps).
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <cerrno>
#include <fstream>
#include <ios>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/bes.h"
#include "bes_launch.h"
#include "bes_status.h"
#ifndef BES_SYSTEM_DEFINITION
#include "km_model.cuh"
#else
#include BES_SYSTEM_DEFINITION
#endif

using bes::DeviceProblem;

namespace {

enum BufId {
    B_TIME_DOMAIN, B_ACTUAL_TIME, B_STATE, B_UPAR, B_SPAR, B_GPAR, B_IGPAR, B_UACC, B_IUACC, B_SACC, B_ISACC,
    B_COUPLING, B_COUPLING_STRENGTH, B_COUPLING_INDEX, B_DENSE_INDEX, B_DENSE_TIME, B_DENSE_STATE,
    B_RTOL, B_ATOL, B_CROW, B_CCOL, B_CNT_ACC, B_CNT_REJ, B_CNT_BICG, B_CNT_RHS, B_STATUS,
    B_PREF, B_PERIOD, B_MAXACC, B_POINCARE,   /* period analysis, allocated by bes_set_period_analysis */
    B_COUNT
};

struct Buf {
    void* h = nullptr;
    void* d = nullptr;
    int64_t count = 0;
    size_t elem = 8;
    size_t bytes() const { return (size_t)count * elem; }
};

thread_local std::string g_create_error;

}  // namespace

struct bes_solver {
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t sync_event = nullptr, t0 = nullptr, t1 = nullptr;
    int n_systems = 0, ud = 0, nup = 0, nsp = 0, ngp = 0, nigp = 0, nua = 0, niua = 0, nsa = 0, nisa = 0, ne = 0,
        ndo = 0, nc = 1, algorithm = 1;
    int cbw = 0, cci = 0;   /* coupling storage of the reference: bandwidth, circular indicator */
    std::vector<int32_t> units;
    std::vector<int64_t> unit_offset;
    int64_t total_units = 0;
    int n_matrices = 1;
    std::vector<int32_t> matrix_of_system, matrix_dim;
    std::vector<char> matrix_symmetric;   /* per matrix, as last copied to the device (exact C == C^T) */
    std::vector<int64_t> matrix_offset, coupling_offset;
    Buf buf[B_COUNT];
    /* device-only metadata */
    int32_t* d_units = nullptr;
    int64_t* d_unit_offset = nullptr;
    int64_t* d_coupling_offset = nullptr;
    int32_t* d_order = nullptr;
    int32_t* h_order = nullptr;
    int32_t* d_work = nullptr;
    double* d_event_tol = nullptr;
    int32_t* d_event_dir = nullptr;
    double* d_uacc_reset = nullptr;
    int32_t* d_iuacc_reset = nullptr;
    std::vector<double> event_tol, uacc_reset;
    std::vector<int32_t> event_dir, iuacc_reset;
    /* options (defaults: Interface.cuh:613-635) */
    double dt0 = 1e-2, dtmax = 1.0e6, dtmin = 1.0e-12, grow = 5.0, shrink = 0.1, do_min_dt = 0.0;
    int active = 0, do_freq = 1, bicg_max_iter = 19, warps_per_block = 0;
    int shared_globals = 1, shared_coupling = 0;
    long long max_steps = 1000000;
    /* launch plan */
    bool order_dirty = true;
    int analysis_sections = -1;   /* -1: per-period analysis off */
    double analysis_tol = 1e-6;
    int analysis_accessory = 0;
    bool scaled_coupling[2] = {false, false};   /* a host copy of CouplingRow/ColumnScale with a value != 1 went to the device */
    int class_begin[3] = {0, 0, 0}, class_count[3] = {0, 0, 0};
    bool class0_all32 = false;
    bool class_shared[3] = {false, false, false};   /* every system of the class uses one matrix */
    bool class_symmetric[3] = {false, false, false}; /* ... and that matrix equals its transpose exactly */
    int sm_count = 148;
    /* the classes run concurrently: fork/join streams, and the whole solve is
     * captured once into a CUDA graph that later calls replay */
    cudaStream_t class_stream[3] = {nullptr, nullptr, nullptr};
    cudaEvent_t fork_ev = nullptr, join_ev[3] = {nullptr, nullptr, nullptr};
    cudaGraphExec_t gexec = nullptr;
    int g_periods = -1, g_reset = -2, g_launches = 0;
    bool graph_dirty = true;
    int use_graph = 1;
    int warps_per_system = 0;   /* 0: multi-warp systems above 32 units; 1: one warp per system */
    int bicg_recurrence = 0;    /* 0: the reference's BiCG recurrence; 1: the single-reduction form */
    int tuned_wpb[3] = {0, 0, 0};      /* per size class, set by bes_autotune (0: not tuned) */
    int tuned_wps[3] = {-1, -1, -1};   /* per size class, set by bes_autotune (-1: not tuned) */
    float last_ms = 0.f;
    int last_launches = 0;
    std::string err;
};

namespace {

bes_status fail(bes_solver* h, bes_status code, const char* fmt, ...) {
    char msg[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(msg, sizeof msg, fmt, ap);
    va_end(ap);
    if (h) h->err = msg; else g_create_error = msg;
    return code;
}

#define CUDA_TRY(h, call)                                                                   \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return fail((h), BES_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                        __FILE__, __LINE__);                                                \
    } while (0)

bool is_int_buf(int id) {
    return id == B_IGPAR || id == B_IUACC || id == B_ISACC || id == B_COUPLING_INDEX || id == B_DENSE_INDEX ||
           id == B_STATUS || id == B_PERIOD;
}

int var_to_buf(int var) {
    switch (var) {
        case BES_TIME_DOMAIN: return B_TIME_DOMAIN;
        case BES_ACTUAL_TIME: return B_ACTUAL_TIME;
        case BES_ACTUAL_STATE: return B_STATE;
        case BES_UNIT_PARAMETERS: return B_UPAR;
        case BES_SYSTEM_PARAMETERS: return B_SPAR;
        case BES_GLOBAL_PARAMETERS: return B_GPAR;
        case BES_INTEGER_GLOBAL_PARAMETERS: return B_IGPAR;
        case BES_UNIT_ACCESSORIES: return B_UACC;
        case BES_INTEGER_UNIT_ACCESSORIES: return B_IUACC;
        case BES_SYSTEM_ACCESSORIES: return B_SACC;
        case BES_INTEGER_SYSTEM_ACCESSORIES: return B_ISACC;
        case BES_COUPLING_MATRIX: return B_COUPLING;
        case BES_COUPLING_STRENGTH: return B_COUPLING_STRENGTH;
        case BES_COUPLING_INDEX: return B_COUPLING_INDEX;
        case BES_DENSE_INDEX: return B_DENSE_INDEX;
        case BES_DENSE_TIME: return B_DENSE_TIME;
        case BES_DENSE_STATE: return B_DENSE_STATE;
        case BES_RELATIVE_TOLERANCE_SYSTEM: return B_RTOL;
        case BES_ABSOLUTE_TOLERANCE_SYSTEM: return B_ATOL;
        case BES_COUPLING_ROW_SCALE: return B_CROW;
        case BES_COUPLING_COLUMN_SCALE: return B_CCOL;
        case BES_POINCARE_SECTIONS: return B_POINCARE;
        case BES_PERIOD_NUMBER: return B_PERIOD;
        case BES_MAXIMUM_ACCESSORY: return B_MAXACC;
        default: return -1;
    }
}

const char* var_name(int var) {
    switch (var) {
        case BES_ALL: return "All";
        case BES_TIME_DOMAIN: return "TimeDomain";
        case BES_ACTUAL_TIME: return "ActualTime";
        case BES_ACTUAL_STATE: return "ActualState";
        case BES_UNIT_PARAMETERS: return "UnitParameters";
        case BES_SYSTEM_PARAMETERS: return "SystemParameters";
        case BES_GLOBAL_PARAMETERS: return "GlobalParameters";
        case BES_INTEGER_GLOBAL_PARAMETERS: return "IntegerGlobalParameters";
        case BES_UNIT_ACCESSORIES: return "UnitAccessories";
        case BES_INTEGER_UNIT_ACCESSORIES: return "IntegerUnitAccessories";
        case BES_SYSTEM_ACCESSORIES: return "SystemAccessories";
        case BES_INTEGER_SYSTEM_ACCESSORIES: return "IntegerSystemAccessories";
        case BES_COUPLING_MATRIX: return "CouplingMatrix";
        case BES_COUPLING_STRENGTH: return "CouplingStrength";
        case BES_COUPLING_INDEX: return "CouplingIndex";
        case BES_DENSE_OUTPUT: return "DenseOutput";
        case BES_DENSE_INDEX: return "DenseIndex";
        case BES_DENSE_TIME: return "DenseTime";
        case BES_DENSE_STATE: return "DenseState";
        case BES_RELATIVE_TOLERANCE_SYSTEM: return "RelativeToleranceSystem";
        case BES_ABSOLUTE_TOLERANCE_SYSTEM: return "AbsoluteToleranceSystem";
        case BES_COUNTERS: return "Counters";
        case BES_COUPLING_ROW_SCALE: return "CouplingRowScale";
        case BES_COUPLING_COLUMN_SCALE: return "CouplingColumnScale";
        case BES_POINCARE_SECTIONS: return "PoincareSections";
        case BES_PERIOD_NUMBER: return "PeriodNumber";
        case BES_MAXIMUM_ACCESSORY: return "MaximumAccessory";
        default: return "unknown";
    }
}

bes_status bound(bes_solver* h, const char* fn, const char* what, long long v, long long lo, long long hi) {
    if (v < lo || v > hi) {
        if (lo > hi) return fail(h, BES_ERR_INDEX, "%s: %s index %lld out of range (acceptable index: none)", fn, what, v);
        return fail(h, BES_ERR_INDEX, "%s: %s index %lld out of range (acceptable index: %lld-%lld)", fn, what, v, lo, hi);
    }
    return BES_OK;
}

int units_class(int n) { return n <= 32 ? 0 : (n <= 64 ? 1 : 2); }

bes_status copy_h2d(bes_solver* h, int id) {
    Buf& b = h->buf[id];
    if (b.count > 0) CUDA_TRY(h, cudaMemcpyAsync(b.d, b.h, b.bytes(), cudaMemcpyHostToDevice, h->stream));
    if (id == B_COUPLING) {
        /* the shared-matrix kernels depend on the symmetry of what the device holds */
        const double* C = (const double*)b.h;
        h->matrix_symmetric.assign(h->n_matrices, 0);
        for (int m = 0; m < h->n_matrices; m++) {
            const int n = h->matrix_dim[m];
            const double* Cm = C + h->matrix_offset[m];
            bool sym = true;
            for (int i = 0; i < n && sym; i++)
                for (int j = i + 1; j < n && sym; j++) sym = Cm[i + (int64_t)j * n] == Cm[j + (int64_t)i * n];
            h->matrix_symmetric[m] = sym;
        }
        h->order_dirty = true;
    }
    if (id == B_CROW || id == B_CCOL) {
        const double* v = (const double*)b.h;
        bool any = false;
        for (int64_t i = 0; i < b.count && !any; i++) any = v[i] != 1.0;
        h->scaled_coupling[id == B_CCOL] = any;
    }
    return BES_OK;
}
bes_status copy_d2h(bes_solver* h, int id) {
    Buf& b = h->buf[id];
    if (b.count > 0) CUDA_TRY(h, cudaMemcpyAsync(b.h, b.d, b.bytes(), cudaMemcpyDeviceToHost, h->stream));
    return BES_OK;
}

void free_all(bes_solver* h) {
    if (!h) return;
    cudaSetDevice(h->device);
    for (auto& b : h->buf) {
        if (b.h) cudaFreeHost(b.h);
        if (b.d) cudaFree(b.d);
        b.h = b.d = nullptr;
    }
    void* dev[] = {h->d_units, h->d_unit_offset, h->d_coupling_offset, h->d_order, h->d_work,
                   h->d_event_tol, h->d_event_dir, h->d_uacc_reset, h->d_iuacc_reset};
    for (void* p : dev)
        if (p) cudaFree(p);
    if (h->h_order) cudaFreeHost(h->h_order);
    if (h->gexec) cudaGraphExecDestroy(h->gexec);
    for (int c = 0; c < 3; c++) {
        if (h->class_stream[c]) cudaStreamDestroy(h->class_stream[c]);
        if (h->join_ev[c]) cudaEventDestroy(h->join_ev[c]);
    }
    if (h->fork_ev) cudaEventDestroy(h->fork_ev);
    if (h->sync_event) cudaEventDestroy(h->sync_event);
    if (h->t0) cudaEventDestroy(h->t0);
    if (h->t1) cudaEventDestroy(h->t1);
    if (h->own_stream) cudaStreamDestroy(h->own_stream);
}

/* processing order: active systems grouped by class, costliest (largest N) first */
bes_status build_order(bes_solver* h) {
    const int nact = std::min(h->active, h->n_systems);
    std::vector<int32_t> idx(nact);
    std::iota(idx.begin(), idx.end(), 0);
    std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) {
        int ca = units_class(h->units[a]), cb = units_class(h->units[b]);
        if (ca != cb) return ca < cb;
        return h->units[a] > h->units[b];
    });
    for (int c = 0; c < 3; c++) { h->class_begin[c] = 0; h->class_count[c] = 0; }
    for (int i = 0; i < nact; i++) h->h_order[i] = idx[i];
    int pos = 0;
    for (int c = 0; c < 3; c++) {
        h->class_begin[c] = pos;
        while (pos < nact && units_class(h->units[idx[pos]]) == c) pos++;
        h->class_count[c] = pos - h->class_begin[c];
    }
    h->class0_all32 = true;
    for (int i = 0; i < h->class_count[0]; i++)
        if (h->units[idx[i]] != 32) h->class0_all32 = false;
    for (int c = 0; c < 3; c++) {
        h->class_shared[c] = h->class_count[c] > 0;
        for (int i = 1; i < h->class_count[c]; i++)
            if (h->matrix_of_system[idx[h->class_begin[c] + i]] != h->matrix_of_system[idx[h->class_begin[c]]])
                h->class_shared[c] = false;
        /* a symmetric shared matrix lets one shared-memory read serve both BiCG products */
        h->class_symmetric[c] = false;
        if (h->class_shared[c]) {
            const int m = h->matrix_of_system[idx[h->class_begin[c]]];
            h->class_symmetric[c] = m < (int)h->matrix_symmetric.size() && h->matrix_symmetric[m];
        }
    }
    if (nact > 0)
        CUDA_TRY(h, cudaMemcpyAsync(h->d_order, h->h_order, sizeof(int32_t) * nact, cudaMemcpyHostToDevice, h->stream));
    h->order_dirty = false;
    h->graph_dirty = true;
    return BES_OK;
}

DeviceProblem make_problem(bes_solver* h) {
    DeviceProblem P;
    std::memset(&P, 0, sizeof P);
    P.n_systems = h->n_systems;
    P.total_units = h->total_units;
    P.units = h->d_units;
    P.unit_offset = h->d_unit_offset;
    P.coupling_offset = h->d_coupling_offset;
    P.coupling = (const double*)h->buf[B_COUPLING].d;
    P.state = (double*)h->buf[B_STATE].d;
    P.upar = (const double*)h->buf[B_UPAR].d;
    P.uacc = (double*)h->buf[B_UACC].d;
    P.iuacc = (int32_t*)h->buf[B_IUACC].d;
    P.spar = (double*)h->buf[B_SPAR].d;
    P.sacc = (double*)h->buf[B_SACC].d;
    P.isacc = (int32_t*)h->buf[B_ISACC].d;
    P.gpar = (double*)h->buf[B_GPAR].d;
    P.igpar = (int32_t*)h->buf[B_IGPAR].d;
    P.time_domain = (double*)h->buf[B_TIME_DOMAIN].d;
    P.actual_time = (double*)h->buf[B_ACTUAL_TIME].d;
    P.rtol = (const double*)h->buf[B_RTOL].d;
    P.coupling_row_scale = (const double*)h->buf[B_CROW].d;
    if (h->analysis_sections >= 0) {
        P.period_ref = (double*)h->buf[B_PREF].d;
        P.period_number = (int32_t*)h->buf[B_PERIOD].d;
        P.period_tol = h->analysis_tol;
        P.max_accessory = (double*)h->buf[B_MAXACC].d;
        P.max_accessory_index = h->analysis_accessory;
        P.n_sections = h->analysis_sections;
        P.poincare = h->analysis_sections > 0 ? (double*)h->buf[B_POINCARE].d : nullptr;
    }
    P.coupling_col_scale = (const double*)h->buf[B_CCOL].d;
    P.atol = (const double*)h->buf[B_ATOL].d;
    P.event_tol = h->d_event_tol;
    P.event_dir = h->d_event_dir;
    P.dt0 = h->dt0;
    P.dtmin = h->dtmin;
    P.dtmax = h->dtmax;
    P.grow = h->grow;
    P.shrink = h->shrink;
    P.algorithm = h->algorithm;
    P.bicg_max_iter = h->bicg_max_iter;
    P.max_steps_per_period = h->max_steps;
    P.ndo = h->ndo;
    P.do_save_frequency = h->do_freq;
    P.do_min_dt = h->do_min_dt;
    P.dense_time = (double*)h->buf[B_DENSE_TIME].d;
    P.dense_state = (double*)h->buf[B_DENSE_STATE].d;
    P.dense_index = (int32_t*)h->buf[B_DENSE_INDEX].d;
    P.n_accepted = (unsigned long long*)h->buf[B_CNT_ACC].d;
    P.n_rejected = (unsigned long long*)h->buf[B_CNT_REJ].d;
    P.n_bicg_iter = (unsigned long long*)h->buf[B_CNT_BICG].d;
    P.n_rhs = (unsigned long long*)h->buf[B_CNT_RHS].d;
    P.status = (int32_t*)h->buf[B_STATUS].d;
    P.uacc_reset = h->d_uacc_reset;
    P.iuacc_reset = h->d_iuacc_reset;
    P.band_width = h->cbw;
    return P;
}

struct ClassLaunch {
    bes::Variant v;
    int grid, wpb;
};

/* launch shape of one class (no stream work: safe before a capture) */
bes_status plan_shape(bes_solver* h, int cls, int warps_per_system, int requested_wpb, ClassLaunch* L) {
    const bes::Variant v = bes::class_variant(cls, h->class0_all32, h->shared_coupling && h->class_shared[cls],
                                         warps_per_system, h->class_symmetric[cls], h->bicg_recurrence, h->cbw);
    const int count = h->class_count[cls];
    if (bes::max_warps_per_block(v) < v.G)
        return fail(h, BES_ERR_CUDA, "solver kernel variant (U=%d, G=%d) does not fit in shared memory", v.U, v.G);
    const int wpb = bes::class_warps_per_block(v, count, h->sm_count, requested_wpb);
    int per_sm = 0;
    CUDA_TRY(h, bes::occupancy(v, wpb, &per_sm));
    if (per_sm < 1)
        return fail(h, BES_ERR_CUDA, "solver kernel (U=%d, G=%d) cannot be resident with %d warps per block", v.U,
                    v.G, wpb);
    const int systems_per_cta = wpb / v.G;
    const int needed = (count + systems_per_cta - 1) / systems_per_cta;
    L->v = v;
    L->wpb = wpb;
    L->grid = std::max(1, std::min(needed, per_sm * h->sm_count));
    return BES_OK;
}

/* the class's launch shape: the autotuner's choice if there is one, else the options */
bes_status plan_class(bes_solver* h, int cls, ClassLaunch* L) {
    return plan_shape(h, cls, h->tuned_wps[cls] >= 0 ? h->tuned_wps[cls] : h->warps_per_system,
                      h->tuned_wpb[cls] > 0 ? h->tuned_wpb[cls] : h->warps_per_block, L);
}

/* the whole solve on stream s: reset the work counters, fork one stream per
 * non-empty class, join back into s */
bes_status enqueue_solve(bes_solver* h, DeviceProblem P, cudaStream_t s, const ClassLaunch* L, int* launches) {
    *launches = 0;
    CUDA_TRY(h, cudaMemsetAsync(h->d_work, 0, sizeof(int32_t) * 4, s));
    CUDA_TRY(h, cudaEventRecord(h->fork_ev, s));
    for (int cls = 0; cls < 3; cls++) {
        if (h->class_count[cls] == 0) continue;
        DeviceProblem Pc = P;
        Pc.order = h->d_order + h->class_begin[cls];
        Pc.n_active = h->class_count[cls];
        Pc.work_counter = h->d_work + cls;
        cudaStream_t cs = h->class_stream[cls];
        CUDA_TRY(h, cudaStreamWaitEvent(cs, h->fork_ev, 0));
        CUDA_TRY(h, bes::launch(L[cls].v, Pc, L[cls].grid, L[cls].wpb, cs));
        CUDA_TRY(h, cudaEventRecord(h->join_ev[cls], cs));
        CUDA_TRY(h, cudaStreamWaitEvent(s, h->join_ev[cls], 0));
        (*launches)++;
    }
    return BES_OK;
}

bes_status check_solver(bes_solver* h) {
    if (!h) return BES_ERR_ARGUMENT;
    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) return fail(h, BES_ERR_CUDA, "cudaSetDevice(%d): %s", h->device, cudaGetErrorString(e));
    return BES_OK;
}

}  // namespace

extern "C" {

const char* bes_status_string(bes_status s) {
    switch (s) {
        case BES_OK: return "ok";
        case BES_ERR_ARGUMENT: return "invalid argument";
        case BES_ERR_INDEX: return "index out of range";
        case BES_ERR_OPTION: return "option or variable not applicable";
        case BES_ERR_CUDA: return "CUDA error";
        case BES_ERR_MEMORY: return "out of memory";
        case BES_ERR_IO: return "input/output error";
        case BES_ERR_MODEL: return "sizes do not match the compiled system definition";
        case BES_ERR_UNSUPPORTED: return "unsupported";
        default: return "unknown status";
    }
}

const char* bes_last_error(const bes_solver* h) { return h ? h->err.c_str() : g_create_error.c_str(); }

bes_status bes_model_info_get(bes_model_info* out) {
    if (!out) return BES_ERR_ARGUMENT;
    std::memset(out, 0, sizeof *out);
    out->unit_dim = BES_MODEL_UD;
    out->n_unit_parameters = BES_MODEL_NUP;
    out->n_system_parameters = BES_MODEL_NSP;
    out->n_global_parameters = BES_MODEL_NGP;
    out->n_int_global_parameters = BES_MODEL_NIGP;
    out->n_unit_accessories = BES_MODEL_NUA;
    out->n_int_unit_accessories = BES_MODEL_NIUA;
    out->n_system_accessories = BES_MODEL_NSA;
    out->n_int_system_accessories = BES_MODEL_NISA;
    out->n_events = BES_MODEL_NE;
    out->max_units_per_system = 128;
    std::snprintf(out->name, sizeof out->name, "%s", BES_MODEL_NAME);
    return BES_OK;
}

bes_status bes_device_count(int32_t* count) {
    if (!count) return BES_ERR_ARGUMENT;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) { *count = 0; return fail(nullptr, BES_ERR_CUDA, "cudaGetDeviceCount: %s", cudaGetErrorString(e)); }
    *count = n;
    return BES_OK;
}

bes_status bes_device_info_get(int32_t device, bes_device_info* out) {
    if (!out) return BES_ERR_ARGUMENT;
    std::memset(out, 0, sizeof *out);
    cudaDeviceProp prop;
    cudaError_t e = cudaGetDeviceProperties(&prop, device);
    if (e != cudaSuccess) return fail(nullptr, BES_ERR_CUDA, "cudaGetDeviceProperties(%d): %s", device, cudaGetErrorString(e));
    std::snprintf(out->name, sizeof out->name, "%s", prop.name);
    out->cc_major = prop.major;
    out->cc_minor = prop.minor;
    out->multiprocessors = prop.multiProcessorCount;
    out->global_memory_bytes = prop.totalGlobalMem;
    return BES_OK;
}

bes_status bes_create(const bes_config* c, bes_solver** out) {
    if (!c || !out) return fail(nullptr, BES_ERR_ARGUMENT, "bes_create: null argument");
    *out = nullptr;
    if (c->n_systems <= 0) return fail(nullptr, BES_ERR_ARGUMENT, "bes_create: n_systems must be positive");
    if (c->unit_dim != BES_MODEL_UD || c->n_unit_parameters != BES_MODEL_NUP ||
        c->n_system_parameters != BES_MODEL_NSP || c->n_global_parameters != BES_MODEL_NGP ||
        c->n_int_global_parameters != BES_MODEL_NIGP || c->n_unit_accessories != BES_MODEL_NUA ||
        c->n_int_unit_accessories != BES_MODEL_NIUA || c->n_system_accessories != BES_MODEL_NSA ||
        c->n_int_system_accessories != BES_MODEL_NISA || c->n_events != BES_MODEL_NE)
        return fail(nullptr, BES_ERR_MODEL,
                    "bes_create: sizes (UD=%d NUP=%d NSP=%d NGP=%d NiGP=%d NUA=%d NiUA=%d NSA=%d NiSA=%d NE=%d) do not "
                    "match the compiled system definition '%s' (UD=%d NUP=%d NSP=%d NGP=%d NiGP=%d NUA=%d NiUA=%d "
                    "NSA=%d NiSA=%d NE=%d)",
                    c->unit_dim, c->n_unit_parameters, c->n_system_parameters, c->n_global_parameters,
                    c->n_int_global_parameters, c->n_unit_accessories, c->n_int_unit_accessories,
                    c->n_system_accessories, c->n_int_system_accessories, c->n_events, BES_MODEL_NAME, BES_MODEL_UD,
                    BES_MODEL_NUP, BES_MODEL_NSP, BES_MODEL_NGP, BES_MODEL_NIGP, BES_MODEL_NUA, BES_MODEL_NIUA,
                    BES_MODEL_NSA, BES_MODEL_NISA, BES_MODEL_NE);
    if (c->coupling_bandwidth < 0 || (c->coupling_circular != 0 && c->coupling_circular != 1))
        return fail(nullptr, BES_ERR_ARGUMENT, "bes_create: coupling bandwidth %d / circular indicator %d invalid",
                    c->coupling_bandwidth, c->coupling_circular);
    if (c->algorithm != BES_RK4 && c->algorithm != BES_RKCK45)
        return fail(nullptr, BES_ERR_ARGUMENT, "bes_create: unknown algorithm %d", c->algorithm);
    if (c->n_dense_output < 0 || c->n_couplings < 1)
        return fail(nullptr, BES_ERR_ARGUMENT, "bes_create: n_dense_output >= 0 and n_couplings >= 1 required");

    bes_solver* h = new bes_solver();
    h->device = c->device;
    h->n_systems = c->n_systems;
    h->ud = c->unit_dim; h->nup = c->n_unit_parameters; h->nsp = c->n_system_parameters;
    h->ngp = c->n_global_parameters; h->nigp = c->n_int_global_parameters; h->nua = c->n_unit_accessories;
    h->niua = c->n_int_unit_accessories; h->nsa = c->n_system_accessories; h->nisa = c->n_int_system_accessories;
    h->ne = c->n_events; h->ndo = c->n_dense_output; h->nc = c->n_couplings; h->algorithm = c->algorithm;
    h->cbw = c->coupling_bandwidth;
    h->cci = c->coupling_circular;
    h->active = c->n_systems;
    h->units.resize(h->n_systems);
    h->unit_offset.resize(h->n_systems);
    int64_t off = 0;
    for (int s = 0; s < h->n_systems; s++) {
        int n = c->units ? c->units[s] : c->units_per_system;
        if (n < 1 || n > 128) {
            delete h;
            return fail(nullptr, BES_ERR_ARGUMENT, "bes_create: system %d has %d units (1..128 supported)", s, n);
        }
        h->units[s] = n;
        h->unit_offset[s] = off;
        off += n;
    }
    h->total_units = off;
    /* coupling matrices */
    h->n_matrices = c->n_coupling_matrices > 0 ? c->n_coupling_matrices : 1;
    h->matrix_of_system.resize(h->n_systems);
    for (int s = 0; s < h->n_systems; s++) {
        int m = c->coupling_matrix_of_system ? c->coupling_matrix_of_system[s]
                                             : (h->n_matrices == h->n_systems ? s : 0);
        if (m < 0 || m >= h->n_matrices) {
            delete h;
            return fail(nullptr, BES_ERR_INDEX, "bes_create: system %d uses coupling matrix %d of %d", s, m, h->n_matrices);
        }
        h->matrix_of_system[s] = m;
    }
    h->matrix_dim.assign(h->n_matrices, 0);
    for (int s = 0; s < h->n_systems; s++) {
        int m = h->matrix_of_system[s];
        if (h->matrix_dim[m] == 0) h->matrix_dim[m] = h->units[s];
        else if (h->matrix_dim[m] != h->units[s]) {
            delete h;
            return fail(nullptr, BES_ERR_ARGUMENT, "bes_create: systems of different size share coupling matrix %d", m);
        }
    }
    for (int m = 0; m < h->n_matrices; m++)
        if (h->matrix_dim[m] == 0) h->matrix_dim[m] = c->units_per_system > 0 ? c->units_per_system : 1;
    h->matrix_offset.resize(h->n_matrices);
    int64_t moff = 0;
    for (int m = 0; m < h->n_matrices; m++) {
        h->matrix_offset[m] = moff;
        moff += (int64_t)h->nc * h->matrix_dim[m] * h->matrix_dim[m];
    }
    h->coupling_offset.resize(h->n_systems);
    for (int s = 0; s < h->n_systems; s++) h->coupling_offset[s] = h->matrix_offset[h->matrix_of_system[s]];

    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) {
        std::string m = cudaGetErrorString(e);
        delete h;
        return fail(nullptr, BES_ERR_CUDA, "bes_create: cudaSetDevice(%d): %s", c->device, m.c_str());
    }
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device) == cudaSuccess && sms > 0)
        h->sm_count = sms;

    const int64_t NS = h->n_systems, TU = h->total_units;
    struct { int id; int64_t count; } sizes[] = {
        {B_TIME_DOMAIN, 2 * NS}, {B_ACTUAL_TIME, NS}, {B_STATE, h->ud * TU}, {B_UPAR, h->nup * TU},
        {B_SPAR, h->nsp * NS}, {B_GPAR, h->ngp}, {B_IGPAR, h->nigp}, {B_UACC, h->nua * TU},
        {B_IUACC, h->niua * TU}, {B_SACC, h->nsa * NS}, {B_ISACC, h->nisa * NS}, {B_COUPLING, moff},
        {B_COUPLING_STRENGTH, h->nc * NS}, {B_COUPLING_INDEX, h->nc}, {B_DENSE_INDEX, NS},
        {B_DENSE_TIME, h->ndo * NS}, {B_DENSE_STATE, (int64_t)h->ndo * h->ud * TU}, {B_RTOL, h->ud * NS},
        {B_ATOL, h->ud * NS}, {B_CROW, TU}, {B_CCOL, TU}, {B_CNT_ACC, NS}, {B_CNT_REJ, NS}, {B_CNT_BICG, NS}, {B_CNT_RHS, NS}, {B_STATUS, NS}};
    size_t total_bytes = 0;
    for (auto& sz : sizes) {
        Buf& b = h->buf[sz.id];
        b.count = sz.count;
        b.elem = is_int_buf(sz.id) ? 4 : 8;
        total_bytes += b.bytes();
    }
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess && total_bytes >= free_b) {
        free_all(h);
        delete h;
        return fail(nullptr, BES_ERR_MEMORY, "bes_create: %zu bytes required, %zu free", total_bytes, free_b);
    }
#define CREATE_TRY(call)                                                                              \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess) {                                                                      \
            std::string m_ = cudaGetErrorString(e_);                                                  \
            free_all(h);                                                                              \
            delete h;                                                                                 \
            return fail(nullptr, e_ == cudaErrorMemoryAllocation ? BES_ERR_MEMORY : BES_ERR_CUDA,    \
                        "bes_create: %s: %s", #call, m_.c_str());                                     \
        }                                                                                             \
    } while (0)
    CREATE_TRY(cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking));
    h->stream = h->own_stream;
    CREATE_TRY(cudaEventCreateWithFlags(&h->sync_event, cudaEventDisableTiming));
    CREATE_TRY(cudaEventCreateWithFlags(&h->fork_ev, cudaEventDisableTiming));
    for (int c = 0; c < 3; c++) {
        CREATE_TRY(cudaStreamCreateWithFlags(&h->class_stream[c], cudaStreamNonBlocking));
        CREATE_TRY(cudaEventCreateWithFlags(&h->join_ev[c], cudaEventDisableTiming));
    }
    CREATE_TRY(cudaEventCreate(&h->t0));
    CREATE_TRY(cudaEventCreate(&h->t1));
    for (auto& b : h->buf) {
        if (b.count <= 0) continue;
        CREATE_TRY(cudaMallocHost(&b.h, b.bytes()));
        std::memset(b.h, 0, b.bytes());
        CREATE_TRY(cudaMalloc(&b.d, b.bytes()));
        CREATE_TRY(cudaMemsetAsync(b.d, 0, b.bytes(), h->stream));
    }
    CREATE_TRY(cudaMalloc(&h->d_units, sizeof(int32_t) * NS));
    CREATE_TRY(cudaMalloc(&h->d_unit_offset, sizeof(int64_t) * NS));
    CREATE_TRY(cudaMalloc(&h->d_coupling_offset, sizeof(int64_t) * NS));
    CREATE_TRY(cudaMalloc(&h->d_order, sizeof(int32_t) * NS));
    CREATE_TRY(cudaMallocHost(&h->h_order, sizeof(int32_t) * NS));
    CREATE_TRY(cudaMalloc(&h->d_work, sizeof(int32_t) * 4));
    CREATE_TRY(cudaMalloc(&h->d_event_tol, sizeof(double) * std::max(1, h->ne)));
    CREATE_TRY(cudaMalloc(&h->d_event_dir, sizeof(int32_t) * std::max(1, h->ne)));
    CREATE_TRY(cudaMalloc(&h->d_uacc_reset, sizeof(double) * std::max(1, h->nua)));
    CREATE_TRY(cudaMalloc(&h->d_iuacc_reset, sizeof(int32_t) * std::max(1, h->niua)));
    CREATE_TRY(cudaMemcpy(h->d_units, h->units.data(), sizeof(int32_t) * NS, cudaMemcpyHostToDevice));
    CREATE_TRY(cudaMemcpy(h->d_unit_offset, h->unit_offset.data(), sizeof(int64_t) * NS, cudaMemcpyHostToDevice));
    CREATE_TRY(cudaMemcpy(h->d_coupling_offset, h->coupling_offset.data(), sizeof(int64_t) * NS, cudaMemcpyHostToDevice));
    /* defaults: tolerances 1e-8 for every component, event tolerance 1e-6, direction 0
     * (Interface.cuh:625-636) */
    double* rt = (double*)h->buf[B_RTOL].h;
    double* at = (double*)h->buf[B_ATOL].h;
    for (int64_t i = 0; i < h->ud * NS; i++) { rt[i] = 1e-8; at[i] = 1e-8; }
    CREATE_TRY(cudaMemcpy(h->buf[B_RTOL].d, rt, h->buf[B_RTOL].bytes(), cudaMemcpyHostToDevice));
    CREATE_TRY(cudaMemcpy(h->buf[B_ATOL].d, at, h->buf[B_ATOL].bytes(), cudaMemcpyHostToDevice));
    /* coupling factors a_i = b_j = 1: every system's matrix is the stored one */
    for (int id : {B_CROW, B_CCOL}) {
        double* v = (double*)h->buf[id].h;
        for (int64_t i = 0; i < TU; i++) v[i] = 1.0;
        CREATE_TRY(cudaMemcpy(h->buf[id].d, v, h->buf[id].bytes(), cudaMemcpyHostToDevice));
    }
    h->event_tol.assign(std::max(1, h->ne), 1e-6);
    h->event_dir.assign(std::max(1, h->ne), 0);
    CREATE_TRY(cudaMemcpy(h->d_event_tol, h->event_tol.data(), sizeof(double) * h->event_tol.size(), cudaMemcpyHostToDevice));
    CREATE_TRY(cudaMemcpy(h->d_event_dir, h->event_dir.data(), sizeof(int32_t) * h->event_dir.size(), cudaMemcpyHostToDevice));
    h->uacc_reset.assign(std::max(1, h->nua), 0.0);
    h->iuacc_reset.assign(std::max(1, h->niua), 0);
    CREATE_TRY(cudaMemcpy(h->d_uacc_reset, h->uacc_reset.data(), sizeof(double) * h->uacc_reset.size(), cudaMemcpyHostToDevice));
    CREATE_TRY(cudaMemcpy(h->d_iuacc_reset, h->iuacc_reset.data(), sizeof(int32_t) * h->iuacc_reset.size(), cudaMemcpyHostToDevice));
    CREATE_TRY(cudaStreamSynchronize(h->stream));
#undef CREATE_TRY
    *out = h;
    return BES_OK;
}

bes_status bes_destroy(bes_solver* h) {
    if (!h) return BES_ERR_ARGUMENT;
    cudaSetDevice(h->device);
    cudaStreamSynchronize(h->stream);
    free_all(h);
    delete h;
    return BES_OK;
}

bes_status bes_solver_option(bes_solver* h, int32_t option, double value) {
    if (!h) return BES_ERR_ARGUMENT;
    switch (option) {
        case BES_OPT_INITIAL_TIME_STEP: h->dt0 = value; break;
        case BES_OPT_ACTIVE_SYSTEMS: {
            int a = (int)value;
            if (a < 0) return fail(h, BES_ERR_ARGUMENT, "SolverOption: ActiveSystems must be >= 0");
            h->active = a;
            h->order_dirty = true;
            break;
        }
        case BES_OPT_MAXIMUM_TIME_STEP: h->dtmax = value; break;
        case BES_OPT_MINIMUM_TIME_STEP: h->dtmin = value; break;
        case BES_OPT_TIME_STEP_GROW_LIMIT: h->grow = value; break;
        case BES_OPT_TIME_STEP_SHRINK_LIMIT: h->shrink = value; break;
        case BES_OPT_DENSE_OUTPUT_MINIMUM_TIME_STEP: h->do_min_dt = value; break;
        case BES_OPT_DENSE_OUTPUT_SAVE_FREQUENCY: h->do_freq = (int)value; break;
        case BES_OPT_SHARED_GLOBAL_VARIABLES: h->shared_globals = value != 0.0; break;
        case BES_OPT_SHARED_COUPLING_MATRICES:
            h->shared_coupling = value != 0.0;
            h->order_dirty = true;
            break;
        case BES_OPT_MAX_STEPS_PER_PERIOD:
            if (!(value >= 1.0)) return fail(h, BES_ERR_ARGUMENT, "SolverOption: MaxStepsPerPeriod must be >= 1");
            h->max_steps = (long long)value;
            break;
        case BES_OPT_BICG_MAX_ITERATIONS:
            if (!(value >= 1.0)) return fail(h, BES_ERR_ARGUMENT, "SolverOption: BiCG iterations must be >= 1");
            h->bicg_max_iter = (int)value;
            break;
        case BES_OPT_WARPS_PER_BLOCK:
            h->warps_per_block = (int)value;
            for (int c = 0; c < 3; c++) h->tuned_wpb[c] = 0;   /* an explicit shape replaces the tuned one */
            break;
        case BES_OPT_USE_CUDA_GRAPH: h->use_graph = value != 0.0; break;
        case BES_OPT_WARPS_PER_SYSTEM:
            if (!(value == 0.0 || value == 1.0))
                return fail(h, BES_ERR_ARGUMENT, "SolverOption: WarpsPerSystem must be 0 (automatic) or 1");
            h->warps_per_system = (int)value;
            for (int c = 0; c < 3; c++) h->tuned_wps[c] = -1;
            break;
        case BES_OPT_BICG_RECURRENCE:
            if (!(value == 0.0 || value == 1.0))
                return fail(h, BES_ERR_ARGUMENT, "SolverOption: BiCGRecurrence must be 0 (reference) or 1 (single reduction)");
            h->bicg_recurrence = (int)value;
            break;
        default:
            return fail(h, BES_ERR_OPTION, "SolverOption: option %d needs an index argument or is not applicable", option);
    }
    h->graph_dirty = true; /* the kernel arguments carry the options */
    return BES_OK;
}

bes_status bes_solver_option_indexed(bes_solver* h, int32_t option, int32_t index, double value) {
    bes_status st = check_solver(h);
    if (st) return st;
    switch (option) {
        case BES_OPT_RELATIVE_TOLERANCE:
        case BES_OPT_ABSOLUTE_TOLERANCE: {
            const bool rel = option == BES_OPT_RELATIVE_TOLERANCE;
            if ((st = bound(h, "SolverOption", rel ? "RelativeTolerance" : "AbsoluteTolerance", index, 0, h->ud - 1)))
                return st;
            Buf& b = h->buf[rel ? B_RTOL : B_ATOL];
            double* row = (double*)b.h + (int64_t)index * h->n_systems;
            for (int s = 0; s < h->n_systems; s++) row[s] = value;
            CUDA_TRY(h, cudaMemcpyAsync((double*)b.d + (int64_t)index * h->n_systems, row,
                                        sizeof(double) * h->n_systems, cudaMemcpyHostToDevice, h->stream));
            /* the host row is a staging buffer of an asynchronous copy: complete it */
            CUDA_TRY(h, cudaStreamSynchronize(h->stream));
            return BES_OK;
        }
        case BES_OPT_EVENT_TOLERANCE:
            if ((st = bound(h, "SolverOption", "EventTolerance", index, 0, h->ne - 1))) return st;
            h->event_tol[index] = value;
            CUDA_TRY(h, cudaMemcpy(h->d_event_tol + index, &h->event_tol[index], sizeof(double), cudaMemcpyHostToDevice));
            return BES_OK;
        case BES_OPT_EVENT_DIRECTION:
            if ((st = bound(h, "SolverOption", "EventDirection", index, 0, h->ne - 1))) return st;
            h->event_dir[index] = (int32_t)value;
            CUDA_TRY(h, cudaMemcpy(h->d_event_dir + index, &h->event_dir[index], sizeof(int32_t), cudaMemcpyHostToDevice));
            return BES_OK;
        default:
            return fail(h, BES_ERR_OPTION, "SolverOption: option %d takes no index or is not applicable", option);
    }
}

/* ---------------- element access ---------------- */

static bes_status unit_index(bes_solver* h, const char* fn, int sid, int uid, int64_t* g) {
    bes_status st;
    if ((st = bound(h, fn, "SystemNumber", sid, 0, h->n_systems - 1))) return st;
    if ((st = bound(h, fn, "UnitNumber", uid, 0, h->units[sid] - 1))) return st;
    *g = h->unit_offset[sid] + uid;
    return BES_OK;
}

static bes_status unit_slot(bes_solver* h, const char* fn, int sid, int uid, int var, int k, void** p, bool* is_int) {
    int64_t g;
    bes_status st = unit_index(h, fn, sid, uid, &g);
    if (st) return st;
    int id, lim;
    switch (var) {
        case BES_ACTUAL_STATE: id = B_STATE; lim = h->ud; break;
        case BES_UNIT_PARAMETERS: id = B_UPAR; lim = h->nup; break;
        case BES_UNIT_ACCESSORIES: id = B_UACC; lim = h->nua; break;
        case BES_INTEGER_UNIT_ACCESSORIES: id = B_IUACC; lim = h->niua; break;
        case BES_COUPLING_ROW_SCALE: id = B_CROW; lim = 1; break;
        case BES_COUPLING_COLUMN_SCALE: id = B_CCOL; lim = 1; break;
        default: return fail(h, BES_ERR_OPTION, "%s: variable %s needs a different argument list", fn, var_name(var));
    }
    if ((st = bound(h, fn, var_name(var), k, 0, lim - 1))) return st;
    Buf& b = h->buf[id];
    int64_t i = (int64_t)k * h->total_units + g;
    *is_int = b.elem == 4;
    *p = (char*)b.h + i * b.elem;
    return BES_OK;
}

static bes_status system_slot(bes_solver* h, const char* fn, int sid, int var, int k, void** p, bool* is_int) {
    bes_status st;
    if ((st = bound(h, fn, "SystemNumber", sid, 0, h->n_systems - 1))) return st;
    int id, lim;
    switch (var) {
        case BES_TIME_DOMAIN: id = B_TIME_DOMAIN; lim = 2; break;
        case BES_ACTUAL_TIME: id = B_ACTUAL_TIME; lim = 1; break;
        case BES_SYSTEM_PARAMETERS: id = B_SPAR; lim = h->nsp; break;
        case BES_SYSTEM_ACCESSORIES: id = B_SACC; lim = h->nsa; break;
        case BES_INTEGER_SYSTEM_ACCESSORIES: id = B_ISACC; lim = h->nisa; break;
        case BES_DENSE_TIME: id = B_DENSE_TIME; lim = h->ndo; break;
        case BES_COUPLING_STRENGTH: id = B_COUPLING_STRENGTH; lim = h->nc; break;
        case BES_RELATIVE_TOLERANCE_SYSTEM: id = B_RTOL; lim = h->ud; break;
        case BES_ABSOLUTE_TOLERANCE_SYSTEM: id = B_ATOL; lim = h->ud; break;
        default: return fail(h, BES_ERR_OPTION, "%s: variable %s needs a different argument list", fn, var_name(var));
    }
    if ((st = bound(h, fn, var_name(var), k, 0, lim - 1))) return st;
    Buf& b = h->buf[id];
    int64_t i = (int64_t)k * h->n_systems + sid;
    *is_int = b.elem == 4;
    *p = (char*)b.h + i * b.elem;
    return BES_OK;
}

static bes_status global_slot(bes_solver* h, const char* fn, int var, int k, void** p, bool* is_int) {
    bes_status st;
    int id, lim;
    switch (var) {
        case BES_GLOBAL_PARAMETERS: id = B_GPAR; lim = h->ngp; break;
        case BES_INTEGER_GLOBAL_PARAMETERS: id = B_IGPAR; lim = h->nigp; break;
        case BES_COUPLING_INDEX: id = B_COUPLING_INDEX; lim = h->nc; break;
        default: return fail(h, BES_ERR_OPTION, "%s: variable %s needs a different argument list", fn, var_name(var));
    }
    if ((st = bound(h, fn, var_name(var), k, 0, lim - 1))) return st;
    Buf& b = h->buf[id];
    *is_int = b.elem == 4;
    *p = (char*)b.h + (int64_t)k * b.elem;
    return BES_OK;
}

static bes_status coupling_slot(bes_solver* h, const char* fn, int n, int var, int row, int col, double** p) {
    if (var != BES_COUPLING_MATRIX)
        return fail(h, BES_ERR_OPTION, "%s: variable %s needs a different argument list", fn, var_name(var));
    bes_status st;
    if ((st = bound(h, fn, "CouplingNumber", n, 0, (long long)h->n_matrices * h->nc - 1))) return st;
    int m = n / h->nc, cn = n % h->nc, dim = h->matrix_dim[m];
    if ((st = bound(h, fn, "Coupling Matrix Row", row, 0, dim - 1))) return st;
    if ((st = bound(h, fn, "Coupling Matrix Col", col, 0, dim - 1))) return st;
    *p = (double*)h->buf[B_COUPLING].h + h->matrix_offset[m] + (int64_t)cn * dim * dim + row + (int64_t)col * dim;
    return BES_OK;
}

static bes_status dense_state_slot(bes_solver* h, const char* fn, int sid, int uid, int var, int comp, int slot,
                                   double** p) {
    if (var != BES_DENSE_STATE)
        return fail(h, BES_ERR_OPTION, "%s: variable %s needs a different argument list", fn, var_name(var));
    int64_t g;
    bes_status st = unit_index(h, fn, sid, uid, &g);
    if (st) return st;
    if ((st = bound(h, fn, "ComponentNumber in dense state", comp, 0, h->ud - 1))) return st;
    if ((st = bound(h, fn, "DenseState", slot, 0, h->ndo - 1))) return st;
    *p = (double*)h->buf[B_DENSE_STATE].h + (int64_t)slot * h->ud * h->total_units + (int64_t)comp * h->total_units + g;
    return BES_OK;
}

static inline void put(void* p, bool is_int, double v) {
    if (is_int) *(int32_t*)p = (int32_t)v; else *(double*)p = v;
}
static inline double get(const void* p, bool is_int) { return is_int ? (double)*(const int32_t*)p : *(const double*)p; }

bes_status bes_set_host_unit(bes_solver* h, int32_t sid, int32_t uid, int32_t var, int32_t k, double v) {
    if (!h) return BES_ERR_ARGUMENT;
    void* p; bool ii;
    bes_status st = unit_slot(h, "SetHost", sid, uid, var, k, &p, &ii);
    if (!st) put(p, ii, v);
    return st;
}
bes_status bes_get_host_unit(bes_solver* h, int32_t sid, int32_t uid, int32_t var, int32_t k, double* v) {
    if (!h || !v) return BES_ERR_ARGUMENT;
    void* p; bool ii;
    bes_status st = unit_slot(h, "GetHost", sid, uid, var, k, &p, &ii);
    if (!st) *v = get(p, ii);
    return st;
}
bes_status bes_set_host_system(bes_solver* h, int32_t sid, int32_t var, int32_t k, double v) {
    if (!h) return BES_ERR_ARGUMENT;
    void* p; bool ii;
    bes_status st = system_slot(h, "SetHost", sid, var, k, &p, &ii);
    if (!st) put(p, ii, v);
    return st;
}
bes_status bes_get_host_system(bes_solver* h, int32_t sid, int32_t var, int32_t k, double* v) {
    if (!h || !v) return BES_ERR_ARGUMENT;
    void* p; bool ii;
    bes_status st = system_slot(h, "GetHost", sid, var, k, &p, &ii);
    if (!st) *v = get(p, ii);
    return st;
}
bes_status bes_set_host_global(bes_solver* h, int32_t var, int32_t k, double v) {
    if (!h) return BES_ERR_ARGUMENT;
    void* p; bool ii;
    bes_status st = global_slot(h, "SetHost", var, k, &p, &ii);
    if (!st) put(p, ii, v);
    return st;
}
bes_status bes_get_host_global(bes_solver* h, int32_t var, int32_t k, double* v) {
    if (!h || !v) return BES_ERR_ARGUMENT;
    void* p; bool ii;
    bes_status st = global_slot(h, "GetHost", var, k, &p, &ii);
    if (!st) *v = get(p, ii);
    return st;
}
/* Banded and circular storage (CBW > 0 and/or CCI = 1, Interface.cuh:1010-1070
 * and ExplicitRungeKutta_Steppers.cuh:586-641): element (row, col) lies on
 * shifted diagonal (col - row + CBW) mod N, which must be below 2 CBW + 1 when
 * CBW > 0; with CCI = 1 one value per diagonal serves every row.  The library
 * keeps the full matrix these formats describe (zero off the band, the
 * circulant copies filled in), so the implicit products -- which in the
 * reference index full storage in every mode, Steppers.cuh:660,692 -- see
 * the coupling the format means. */
bes_status bes_set_host_coupling(bes_solver* h, int32_t n, int32_t var, int32_t row, int32_t col, double v) {
    if (!h) return BES_ERR_ARGUMENT;
    double* p;
    bes_status st = coupling_slot(h, "SetHost", n, var, row, col, &p);
    if (st) return st;
    if (h->cbw == 0 && h->cci == 0) {
        *p = v;
        return BES_OK;
    }
    const int m = n / h->nc, dim = h->matrix_dim[m];
    const int d = ((col - row + h->cbw) % dim + dim) % dim;
    if (h->cbw > 0 && d > 2 * h->cbw)
        return fail(h, BES_ERR_INDEX, "SetHost: coupling element (%d, %d) lies outside the band of width %d", row, col,
                    h->cbw);
    if (h->cci == 0) {
        *p = v;
        return BES_OK;
    }
    double* base = p - (row + (int64_t)col * dim);   /* the matrix's (0, 0) */
    for (int r = 0; r < dim; r++) {
        const int c = ((r + col - row) % dim + dim) % dim;
        base[r + (int64_t)c * dim] = v;
    }
    return BES_OK;
}
bes_status bes_get_host_coupling(bes_solver* h, int32_t n, int32_t var, int32_t row, int32_t col, double* v) {
    if (!h || !v) return BES_ERR_ARGUMENT;
    double* p;
    bes_status st = coupling_slot(h, "GetHost", n, var, row, col, &p);
    if (!st) *v = *p;
    return st;
}
bes_status bes_set_host_dense_index(bes_solver* h, int32_t sid, int32_t var, double v) {
    if (!h) return BES_ERR_ARGUMENT;
    if (var != BES_DENSE_INDEX) return fail(h, BES_ERR_OPTION, "SetHost: variable %s needs a different argument list", var_name(var));
    bes_status st = bound(h, "SetHost", "SystemNumber", sid, 0, h->n_systems - 1);
    if (!st) ((int32_t*)h->buf[B_DENSE_INDEX].h)[sid] = (int32_t)v;
    return st;
}
bes_status bes_get_host_dense_index(bes_solver* h, int32_t sid, int32_t var, double* v) {
    if (!h || !v) return BES_ERR_ARGUMENT;
    if (var != BES_DENSE_INDEX) return fail(h, BES_ERR_OPTION, "GetHost: variable %s needs a different argument list", var_name(var));
    bes_status st = bound(h, "GetHost", "SystemNumber", sid, 0, h->n_systems - 1);
    if (!st) *v = ((int32_t*)h->buf[B_DENSE_INDEX].h)[sid];
    return st;
}
bes_status bes_set_host_dense_state(bes_solver* h, int32_t sid, int32_t uid, int32_t var, int32_t comp, int32_t slot, double v) {
    if (!h) return BES_ERR_ARGUMENT;
    double* p;
    bes_status st = dense_state_slot(h, "SetHost", sid, uid, var, comp, slot, &p);
    if (!st) *p = v;
    return st;
}
bes_status bes_get_host_dense_state(bes_solver* h, int32_t sid, int32_t uid, int32_t var, int32_t comp, int32_t slot, double* v) {
    if (!h || !v) return BES_ERR_ARGUMENT;
    double* p;
    bes_status st = dense_state_slot(h, "GetHost", sid, uid, var, comp, slot, &p);
    if (!st) *v = *p;
    return st;
}

/* ---------------- bulk access ---------------- */

bes_status bes_array_size(bes_solver* h, int32_t var, int64_t* count) {
    if (!h || !count) return BES_ERR_ARGUMENT;
    int id = var_to_buf(var);
    if (id < 0) return fail(h, BES_ERR_OPTION, "bes_array_size: variable %s has no single array", var_name(var));
    *count = h->buf[id].count;
    return BES_OK;
}

bes_status bes_set_array(bes_solver* h, int32_t var, const void* src, int64_t count) {
    if (!h || (!src && count > 0)) return BES_ERR_ARGUMENT;
    int id = var_to_buf(var);
    if (id < 0) return fail(h, BES_ERR_OPTION, "bes_set_array: variable %s has no single array", var_name(var));
    Buf& b = h->buf[id];
    if (count != b.count)
        return fail(h, BES_ERR_ARGUMENT, "bes_set_array(%s): %lld elements given, %lld expected", var_name(var),
                    (long long)count, (long long)b.count);
    if (count > 0) std::memcpy(b.h, src, b.bytes());
    return BES_OK;
}

bes_status bes_get_array(bes_solver* h, int32_t var, void* dst, int64_t count) {
    if (!h || (!dst && count > 0)) return BES_ERR_ARGUMENT;
    int id = var_to_buf(var);
    if (id < 0) return fail(h, BES_ERR_OPTION, "bes_get_array: variable %s has no single array", var_name(var));
    Buf& b = h->buf[id];
    if (count != b.count)
        return fail(h, BES_ERR_ARGUMENT, "bes_get_array(%s): %lld elements requested, %lld available", var_name(var),
                    (long long)count, (long long)b.count);
    if (count > 0) std::memcpy(dst, b.h, b.bytes());
    return BES_OK;
}

/* ---------------- transfers ---------------- */

static bes_status transfer(bes_solver* h, int32_t var, bool to_device) {
    bes_status st = check_solver(h);
    if (st) return st;
    auto one = [&](int id) { return to_device ? copy_h2d(h, id) : copy_d2h(h, id); };
    switch (var) {
        case BES_ALL: {
            const int ids[] = {B_TIME_DOMAIN, B_ACTUAL_TIME, B_STATE, B_UPAR, B_SPAR, B_GPAR, B_IGPAR, B_UACC,
                               B_IUACC, B_SACC, B_ISACC, B_COUPLING, B_COUPLING_STRENGTH, B_COUPLING_INDEX,
                               B_DENSE_INDEX, B_DENSE_TIME, B_DENSE_STATE, B_RTOL, B_ATOL, B_CROW, B_CCOL};
            for (int id : ids)
                if ((st = one(id))) return st;
            if (!to_device) {
                const int cids[] = {B_CNT_ACC, B_CNT_REJ, B_CNT_BICG, B_CNT_RHS, B_STATUS};
                for (int id : cids)
                    if ((st = one(id))) return st;
            }
            return BES_OK;
        }
        case BES_DENSE_OUTPUT:
            if ((st = one(B_DENSE_INDEX))) return st;
            if ((st = one(B_DENSE_TIME))) return st;
            return one(B_DENSE_STATE);
        case BES_COUNTERS: {
            const int cids[] = {B_CNT_ACC, B_CNT_REJ, B_CNT_BICG, B_CNT_RHS, B_STATUS};
            for (int id : cids)
                if ((st = one(id))) return st;
            return BES_OK;
        }
        default: {
            int id = var_to_buf(var);
            if (id < 0 || var == BES_DENSE_INDEX || var == BES_DENSE_TIME || var == BES_DENSE_STATE)
                return fail(h, BES_ERR_OPTION, "Synchronise%s: variable %s is not applicable",
                            to_device ? "FromHostToDevice" : "FromDeviceToHost", var_name(var));
            return one(id);
        }
    }
}

bes_status bes_synchronise_host_to_device(bes_solver* h, int32_t var) { return transfer(h, var, true); }
bes_status bes_synchronise_device_to_host(bes_solver* h, int32_t var) { return transfer(h, var, false); }

/* ---------------- execution ---------------- */

bes_status bes_set_accessory_reset(bes_solver* h, const double* uacc, const int32_t* iuacc) {
    bes_status st = check_solver(h);
    if (st) return st;
    if (h->nua > 0 && uacc) {
        std::memcpy(h->uacc_reset.data(), uacc, sizeof(double) * h->nua);
        CUDA_TRY(h, cudaMemcpy(h->d_uacc_reset, h->uacc_reset.data(), sizeof(double) * h->nua, cudaMemcpyHostToDevice));
    }
    if (h->niua > 0 && iuacc) {
        std::memcpy(h->iuacc_reset.data(), iuacc, sizeof(int32_t) * h->niua);
        CUDA_TRY(h, cudaMemcpy(h->d_iuacc_reset, h->iuacc_reset.data(), sizeof(int32_t) * h->niua, cudaMemcpyHostToDevice));
    }
    return BES_OK;
}

bes_status bes_solve_periods(bes_solver* h, int32_t n_periods, int32_t reset_at) {
    bes_status st = check_solver(h);
    if (st) return st;
    if (n_periods < 0) return fail(h, BES_ERR_ARGUMENT, "bes_solve_periods: n_periods must be >= 0");
    if (h->order_dirty && (st = build_order(h))) return st;
    DeviceProblem P = make_problem(h);
    P.n_periods = n_periods;
    P.reset_at = reset_at;
    ClassLaunch L[3] = {};
    for (int cls = 0; cls < 3; cls++)
        if (h->class_count[cls] > 0 && (st = plan_class(h, cls, &L[cls]))) return st;
    if (h->scaled_coupling[0] || h->scaled_coupling[1])
        for (int cls = 0; cls < 3; cls++)
            if (h->class_count[cls] > 0 && L[cls].v.rhs < 3)
                return fail(h, BES_ERR_ARGUMENT,
                            "bes_solve_periods: CouplingRowScale / CouplingColumnScale hold values other than 1, "
                            "which only the shared-matrix kernels apply: turn SharedCouplingMatrices on and give "
                            "every system of a size class the same matrix (systems of more than 32 units)");
    if (!h->use_graph) {
        CUDA_TRY(h, cudaEventRecord(h->t0, h->stream));
        if ((st = enqueue_solve(h, P, h->stream, L, &h->last_launches))) return st;
        CUDA_TRY(h, cudaEventRecord(h->t1, h->stream));
        return BES_OK;
    }
    if (h->graph_dirty || h->gexec == nullptr || h->g_periods != n_periods || h->g_reset != reset_at) {
        /* capture on the solver's own stream; the graph is replayed on the caller's */
        if (h->gexec) { cudaGraphExecDestroy(h->gexec); h->gexec = nullptr; }
        CUDA_TRY(h, cudaStreamSynchronize(h->own_stream));
        CUDA_TRY(h, cudaStreamBeginCapture(h->own_stream, cudaStreamCaptureModeThreadLocal));
        int launches = 0;
        st = enqueue_solve(h, P, h->own_stream, L, &launches);
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamEndCapture(h->own_stream, &graph);
        if (st) { if (graph) cudaGraphDestroy(graph); return st; }
        if (e != cudaSuccess) return fail(h, BES_ERR_CUDA, "cudaStreamEndCapture: %s", cudaGetErrorString(e));
        e = cudaGraphInstantiate(&h->gexec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) return fail(h, BES_ERR_CUDA, "cudaGraphInstantiate: %s", cudaGetErrorString(e));
        h->g_periods = n_periods;
        h->g_reset = reset_at;
        h->g_launches = launches;
        h->graph_dirty = false;
    }
    CUDA_TRY(h, cudaEventRecord(h->t0, h->stream));
    CUDA_TRY(h, cudaGraphLaunch(h->gexec, h->stream));
    CUDA_TRY(h, cudaEventRecord(h->t1, h->stream));
    h->last_launches = h->g_launches;
    return BES_OK;
}

bes_status bes_solve(bes_solver* h) { return bes_solve_periods(h, 1, -1); }

/* ---------------- per-period analysis and output files ---------------- */

bes_status bes_set_period_analysis(bes_solver* h, int32_t sections, double distance_tolerance,
                                   int32_t accessory_index) {
    bes_status st = check_solver(h);
    if (st) return st;
    if (sections >= 0 && !(distance_tolerance >= 0.0))
        return fail(h, BES_ERR_ARGUMENT, "bes_set_period_analysis: distance tolerance must be >= 0");
    if (sections >= 0 && (accessory_index < 0 || accessory_index >= std::max(1, h->nua)))
        return fail(h, BES_ERR_INDEX, "bes_set_period_analysis: accessory index %d out of range (0-%d)",
                    accessory_index, std::max(1, h->nua) - 1);
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    for (int id : {B_PREF, B_PERIOD, B_MAXACC, B_POINCARE}) {
        Buf& b = h->buf[id];
        if (b.h) cudaFreeHost(b.h);
        if (b.d) cudaFree(b.d);
        b.h = b.d = nullptr;
        b.count = 0;
    }
    h->analysis_sections = -1;
    h->graph_dirty = true;
    if (sections < 0) return BES_OK;
    const int64_t TU = h->total_units;
    const struct { int id; int64_t count; } sizes[] = {
        {B_PREF, h->ud * TU}, {B_PERIOD, TU}, {B_MAXACC, TU}, {B_POINCARE, (int64_t)sections * TU}};
    for (auto& sz : sizes) {
        Buf& b = h->buf[sz.id];
        b.count = sz.count;
        b.elem = is_int_buf(sz.id) ? 4 : 8;
        if (b.count <= 0) continue;
        cudaError_t e = cudaMallocHost(&b.h, b.bytes());
        if (e == cudaSuccess) e = cudaMalloc(&b.d, b.bytes());
        if (e == cudaSuccess) e = cudaMemsetAsync(b.d, 0, b.bytes(), h->stream);
        if (e != cudaSuccess) {
            bes_set_period_analysis(h, -1, 0.0, 0);
            return fail(h, BES_ERR_MEMORY, "bes_set_period_analysis: %lld sections of %lld units: %s",
                        (long long)sections, (long long)TU, cudaGetErrorString(e));
        }
        std::memset(b.h, 0, b.bytes());
    }
    h->analysis_sections = sections;
    h->analysis_tol = distance_tolerance;
    h->analysis_accessory = accessory_index;
    return BES_OK;
}

/* Print(var) / Print(var, n) of the reference (Interface.cuh:1809-1947 with
 * its writers :1530-1805): the host mirror of a variable to
 * <Name>InSolverObject.txt (CouplingMatrix: ..._<n>.txt; DenseOutput:
 * DenseOutput_<system>.txt with the system's parameters, accessories and time
 * series), every value in width 18, scientific with 10 digits, followed by a
 * comma.  The unit-scope files have one row per unit (no thread padding
 * rows: the library stores none). */
bes_status bes_print(bes_solver* h, int32_t var, int32_t serial, const char* directory) {
    bes_status st = check_solver(h);
    if (st) return st;
    const std::string dir = directory && directory[0] ? std::string(directory) + "/" : std::string();
    const int W = 18;
    auto open = [&](const std::string& name, std::ofstream& f) -> bool {
        f.open(dir + name);
        f.precision(10);
        f.flags(std::ios::scientific);
        return (bool)f;
    };
    auto value = [&](std::ofstream& f, int id, int64_t k) {
        f.width(W);
        if (is_int_buf(id)) f << ((const int32_t*)h->buf[id].h)[k];
        else f << ((const double*)h->buf[id].h)[k];
    };
    const int64_t NS = h->n_systems, TU = h->total_units;
    if (var == BES_COUPLING_MATRIX) {
        if ((st = bound(h, "Print", "CouplingMatrix", serial, 0, (long long)h->n_matrices * h->nc - 1))) return st;
        const int m = serial / h->nc, cn = serial % h->nc, n = h->matrix_dim[m];
        std::ofstream f;
        if (!open("CouplingMatrixInSolverObject_" + std::to_string(serial) + ".txt", f))
            return fail(h, BES_ERR_IO, "Print: cannot open the coupling matrix file in '%s'", dir.c_str());
        const int64_t base = h->matrix_offset[m] + (int64_t)cn * n * n;
        for (int i = 0; i < n; i++) {
            for (int j = 0; j < n; j++) { value(f, B_COUPLING, base + i + (int64_t)j * n); f << ','; }
            f << '\n';
        }
        return f ? BES_OK : fail(h, BES_ERR_IO, "Print: writing the coupling matrix failed");
    }
    if (var == BES_DENSE_OUTPUT) {
        if ((st = bound(h, "Print", "DenseOutput", serial, 0, NS - 1))) return st;
        std::ofstream f;
        if (!open("DenseOutput_" + std::to_string(serial) + ".txt", f))
            return fail(h, BES_ERR_IO, "Print: cannot open the dense output file in '%s'", dir.c_str());
        const int n = h->units[serial];
        const int64_t off = h->unit_offset[serial];
        auto unit_block = [&](const char* title, int id, int count) {
            f << title << ":\n";
            f.width(W); f << "Serial No." << ',';
            for (int u = 0; u < n; u++) { f.width(W); f << "U" + std::to_string(u); if (u < n - 1) f << ','; }
            f << '\n';
            for (int k = 0; k < count; k++) {
                f.width(W); f << k << ',';
                for (int u = 0; u < n; u++) { value(f, id, (int64_t)k * TU + off + u); if (u < n - 1) f << ','; }
                f << '\n';
            }
            f << '\n';
        };
        auto row_block = [&](const char* title, int id, int count, int64_t stride, int64_t first) {
            f << title << ":\n";
            for (int k = 0; k < count; k++) { value(f, id, first + (int64_t)k * stride); if (k < count - 1) f << ','; }
            f << '\n' << '\n';
        };
        unit_block("UnitParameters", B_UPAR, h->nup);
        unit_block("UnitAccessories", B_UACC, h->nua);
        unit_block("IntegerUnitAccessories", B_IUACC, h->niua);
        row_block("SystemParameters", B_SPAR, h->nsp, NS, serial);
        row_block("SystemAccessories", B_SACC, h->nsa, NS, serial);
        row_block("IntegerSystemAccessories", B_ISACC, h->nisa, NS, serial);
        row_block("GlobalParameters", B_GPAR, h->ngp, 1, 0);
        row_block("IntegerGlobalParameters", B_IGPAR, h->nigp, 1, 0);
        f << "Time series:\n";
        f.width(W); f << "t" << ',';
        for (int u = 0; u < n; u++)
            for (int c = 0; c < h->ud; c++) {
                f.width(W); f << "U" + std::to_string(u) + "/C" + std::to_string(c);
                if (u < n - 1 || c < h->ud - 1) f << ',';
            }
        f << '\n';
        const int rows = h->ndo > 0 ? std::min(((const int32_t*)h->buf[B_DENSE_INDEX].h)[serial], h->ndo) : 0;
        for (int i = 0; i < rows; i++) {
            value(f, B_DENSE_TIME, (int64_t)i * NS + serial);
            f << ',';
            for (int u = 0; u < n; u++)
                for (int c = 0; c < h->ud; c++) {
                    value(f, B_DENSE_STATE, (int64_t)i * h->ud * TU + (int64_t)c * TU + off + u);
                    if (u < n - 1 || c < h->ud - 1) f << ',';
                }
            f << '\n';
        }
        return f ? BES_OK : fail(h, BES_ERR_IO, "Print: writing the dense output failed");
    }
    int id = -1;
    int64_t rows = 0, cols = 0;
    switch (var) {
        case BES_TIME_DOMAIN: id = B_TIME_DOMAIN; rows = NS; cols = 2; break;
        case BES_ACTUAL_TIME: id = B_ACTUAL_TIME; rows = NS; cols = 1; break;
        case BES_ACTUAL_STATE: id = B_STATE; rows = TU; cols = h->ud; break;
        case BES_UNIT_PARAMETERS: id = B_UPAR; rows = TU; cols = h->nup; break;
        case BES_SYSTEM_PARAMETERS: id = B_SPAR; rows = NS; cols = h->nsp; break;
        case BES_GLOBAL_PARAMETERS: id = B_GPAR; rows = h->ngp; cols = 1; break;
        case BES_INTEGER_GLOBAL_PARAMETERS: id = B_IGPAR; rows = h->nigp; cols = 1; break;
        case BES_UNIT_ACCESSORIES: id = B_UACC; rows = TU; cols = h->nua; break;
        case BES_INTEGER_UNIT_ACCESSORIES: id = B_IUACC; rows = TU; cols = h->niua; break;
        case BES_SYSTEM_ACCESSORIES: id = B_SACC; rows = NS; cols = h->nsa; break;
        case BES_INTEGER_SYSTEM_ACCESSORIES: id = B_ISACC; rows = NS; cols = h->nisa; break;
        case BES_COUPLING_STRENGTH: id = B_COUPLING_STRENGTH; rows = NS; cols = h->nc; break;
        case BES_COUPLING_INDEX: id = B_COUPLING_INDEX; rows = h->nc; cols = 1; break;
        default:
            return fail(h, BES_ERR_OPTION, "Print: option %s needs a different argument list or is not applicable",
                        var_name(var));
    }
    std::ofstream f;
    if (!open(std::string(var_name(var)) + "InSolverObject.txt", f))
        return fail(h, BES_ERR_IO, "Print: cannot open the file for %s in '%s'", var_name(var), dir.c_str());
    for (int64_t i = 0; i < rows; i++) {
        for (int64_t j = 0; j < cols; j++) { value(f, id, i + j * rows); f << ','; }
        f << '\n';
    }
    return f ? BES_OK : fail(h, BES_ERR_IO, "Print: writing %s failed", var_name(var));
}

/* The reference drivers' output files, written from the host mirrors (call
 * bes_synchronise_device_to_host for the variables first):
 *   BES_CSV_COLLAPSE   CollapseStrength.cu:174-198  (per system and record slot: id, uPAR15, uPAR16,
 *                      every unit's uACC[slot], every unit's uACC[slot + NUA/2])
 *   BES_CSV_POINCARE   BubbleEnsemble.cu:435-455    (per stored section and system: id, uPAR15, R/R_E per unit)
 *   BES_CSV_PERIOD     BubbleEnsemble.cu:457-473    (per system: id, uPAR15, period number per unit)
 *   BES_CSV_EXPANSION  BubbleEnsemble.cu:475-491    (per system: id, uPAR16, the maximum accessory per unit,
 *                      truncated to an integer as the reference's int array stores it)
 * with the reference's stream widths, precisions and scientific notation. */
bes_status bes_write_csv(bes_solver* h, int32_t kind, const char* path) {
    bes_status st = check_solver(h);
    if (st) return st;
    if (!path) return fail(h, BES_ERR_ARGUMENT, "bes_write_csv: path is NULL");
    if (h->nup < 17) return fail(h, BES_ERR_MODEL, "bes_write_csv: the system definition has fewer than 17 unit parameters");
    if ((kind == BES_CSV_POINCARE || kind == BES_CSV_PERIOD || kind == BES_CSV_EXPANSION) && h->analysis_sections < 0)
        return fail(h, BES_ERR_ARGUMENT, "bes_write_csv: per-period analysis is off (bes_set_period_analysis)");
    if (kind == BES_CSV_COLLAPSE && (h->nua < 2 || h->nua % 2))
        return fail(h, BES_ERR_MODEL, "bes_write_csv: the collapse file needs an even number of unit accessories");
    if (kind < BES_CSV_COLLAPSE || kind > BES_CSV_EXPANSION)
        return fail(h, BES_ERR_ARGUMENT, "bes_write_csv: unknown kind %d", kind);
    std::ofstream f(path);
    if (!f) return fail(h, BES_ERR_IO, "bes_write_csv: cannot open %s", path);
    f.flags(std::ios::scientific);
    const double* up = (const double*)h->buf[B_UPAR].h;
    const int64_t TU = h->total_units;
    auto upar = [&](int s, int k) { return up[(int64_t)k * TU + h->unit_offset[s]]; };
    if (kind == BES_CSV_COLLAPSE) {
        const double* ua = (const double*)h->buf[B_UACC].h;
        const int ncoll = h->nua / 2;
        for (int s = 0; s < h->n_systems; s++) {
            const int64_t off = h->unit_offset[s];
            for (int c = 0; c < ncoll; c++) {
                f.width(6); f << s << ',';
                f.width(17); f.precision(10); f << upar(s, 15) << ',';
                f.width(17); f.precision(10); f << upar(s, 16) << ',';
                for (int u = 0; u < h->units[s]; u++) {
                    f.width(10); f.precision(3); f << ua[(int64_t)c * TU + off + u] << ',';
                }
                for (int u = 0; u < h->units[s]; u++) {
                    f.width(10); f.precision(3); f << ua[(int64_t)(c + ncoll) * TU + off + u] << ',';
                }
                f << '\n';
            }
        }
    } else {
        f.precision(10);
        const int W = 18;
        const int nsec = kind == BES_CSV_POINCARE ? h->analysis_sections : 1;
        for (int k = 0; k < nsec; k++) {
            for (int s = 0; s < h->n_systems; s++) {
                const int64_t off = h->unit_offset[s];
                f.width(4); f << s << ',';
                f.width(W); f << upar(s, kind == BES_CSV_EXPANSION ? 16 : 15) << ',';
                for (int u = 0; u < h->units[s]; u++) {
                    if (kind == BES_CSV_POINCARE) {
                        f.width(W); f << ((const double*)h->buf[B_POINCARE].h)[(int64_t)k * TU + off + u] << ',';
                    } else if (kind == BES_CSV_PERIOD) {
                        f.width(4); f << ((const int32_t*)h->buf[B_PERIOD].h)[off + u] << ',';
                    } else {
                        /* truncation toward zero as the reference's int array; non-finite or out
                         * of the int range (undefined for a plain cast) print 0 */
                        const double a = ((const double*)h->buf[B_MAXACC].h)[off + u];
                        const int t = (std::isfinite(a) && std::fabs(a) < 2147483647.0) ? (int)a : 0;
                        f.width(4); f << t << ',';
                    }
                }
                f << '\n';
            }
        }
    }
    if (!f) return fail(h, BES_ERR_IO, "bes_write_csv: writing %s failed", path);
    return BES_OK;
}

/* Launch-shape autotuner: for every non-empty size class, time each launch
 * shape the kernels allow (warps per system, then warps per CTA in powers of
 * two up to what shared memory and the launch bounds admit) on the device's
 * current inputs, from the same saved state each time, and keep the fastest.
 * Every shape computes bit-identical results, so the choice changes speed
 * only.  The state, accessories, dense output and counters on the device are
 * restored afterwards; the host mirrors are not touched. */
bes_status bes_autotune(bes_solver* h, int32_t n_periods, int64_t step_cap, bes_autotune_result* result) {
    bes_status st = check_solver(h);
    if (st) return st;
    if (!result) return fail(h, BES_ERR_ARGUMENT, "bes_autotune: result is NULL");
    std::memset(result, 0, sizeof(*result));
    if (n_periods < 1) n_periods = 1;
    if (h->order_dirty && (st = build_order(h))) return st;
    const int saved[] = {B_TIME_DOMAIN, B_ACTUAL_TIME, B_STATE, B_UACC, B_IUACC, B_SACC, B_ISACC, B_DENSE_INDEX,
                         B_DENSE_TIME, B_DENSE_STATE, B_CNT_ACC, B_CNT_REJ, B_CNT_BICG, B_CNT_RHS, B_STATUS};
    constexpr int NSAVED = sizeof(saved) / sizeof(saved[0]);
    void* backup[NSAVED] = {};
    auto release = [&]() {
        for (void*& p : backup)
            if (p) { cudaFree(p); p = nullptr; }
    };
    auto restore = [&]() -> cudaError_t {
        for (int k = 0; k < NSAVED; k++) {
            const Buf& b = h->buf[saved[k]];
            if (b.count <= 0) continue;
            cudaError_t e = cudaMemcpyAsync(b.d, backup[k], b.bytes(), cudaMemcpyDeviceToDevice, h->stream);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    };
    for (int k = 0; k < NSAVED; k++) {
        const Buf& b = h->buf[saved[k]];
        if (b.count <= 0) continue;
        cudaError_t e = cudaMalloc(&backup[k], b.bytes());
        if (e == cudaSuccess) e = cudaMemcpyAsync(backup[k], b.d, b.bytes(), cudaMemcpyDeviceToDevice, h->stream);
        if (e != cudaSuccess) {
            release();
            return fail(h, BES_ERR_MEMORY, "bes_autotune: saving the device state: %s", cudaGetErrorString(e));
        }
    }
    DeviceProblem P = make_problem(h);
    P.n_periods = n_periods;
    P.reset_at = -1;
    if (step_cap > 0) P.max_steps_per_period = std::min<int64_t>(P.max_steps_per_period, step_cap);
    for (int cls = 0; cls < 3 && !st; cls++) {
        if (h->class_count[cls] == 0) continue;
        float best = -1.0f;
        int best_wps = 0, best_wpb = 0;
        for (int wps = 0; wps <= (cls == 0 ? 0 : 1) && !st; wps++) {
            const bes::Variant v = bes::class_variant(cls, h->class0_all32,
                                                      h->shared_coupling && h->class_shared[cls], wps,
                                                      h->class_symmetric[cls], h->bicg_recurrence, h->cbw);
            const int cap = bes::max_warps_per_block(v);
            for (int wpb = v.G; wpb <= cap && !st; wpb *= 2) {
                ClassLaunch L;
                if ((st = plan_shape(h, cls, wps, wpb, &L))) break;
                if (L.wpb != wpb) continue;   /* clamped to a shape already timed */
                DeviceProblem Pc = P;
                Pc.order = h->d_order + h->class_begin[cls];
                Pc.n_active = h->class_count[cls];
                Pc.work_counter = h->d_work + cls;
                cudaError_t e = restore();
                if (e == cudaSuccess) e = cudaMemsetAsync(h->d_work, 0, sizeof(int32_t) * 4, h->stream);
                if (e == cudaSuccess) e = cudaEventRecord(h->t0, h->stream);
                if (e == cudaSuccess) e = bes::launch(L.v, Pc, L.grid, L.wpb, h->stream);
                if (e == cudaSuccess) e = cudaEventRecord(h->t1, h->stream);
                if (e == cudaSuccess) e = cudaEventSynchronize(h->t1);
                float ms = 0.0f;
                if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, h->t0, h->t1);
                if (e != cudaSuccess) {
                    st = fail(h, BES_ERR_CUDA, "bes_autotune: class %d, %d warps per system, %d per CTA: %s", cls,
                              wps, wpb, cudaGetErrorString(e));
                    break;
                }
                result->candidates++;
                if (best < 0.0f || ms < best) { best = ms; best_wps = wps; best_wpb = L.wpb; }
            }
        }
        if (!st) {
            h->tuned_wps[cls] = best_wps;
            h->tuned_wpb[cls] = best_wpb;
            result->warps_per_system[cls] = best_wps;
            result->warps_per_block[cls] = best_wpb;
            result->ms[cls] = best;
        }
    }
    cudaError_t e = restore();
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    release();
    h->graph_dirty = true;
    if (st) return st;
    if (e != cudaSuccess) return fail(h, BES_ERR_CUDA, "bes_autotune: restoring the device state: %s", cudaGetErrorString(e));
    return BES_OK;
}

bes_status bes_synchronise_device(bes_solver* h) {
    bes_status st = check_solver(h);
    if (st) return st;
    CUDA_TRY(h, cudaDeviceSynchronize());
    return BES_OK;
}

bes_status bes_insert_synchronisation_point(bes_solver* h) {
    bes_status st = check_solver(h);
    if (st) return st;
    CUDA_TRY(h, cudaEventRecord(h->sync_event, h->stream));
    return BES_OK;
}

bes_status bes_synchronise_solver(bes_solver* h) {
    bes_status st = check_solver(h);
    if (st) return st;
    CUDA_TRY(h, cudaEventSynchronize(h->sync_event));
    CUDA_TRY(h, cudaGetLastError());
    return BES_OK;
}

bes_status bes_set_stream(bes_solver* h, void* cuda_stream) {
    bes_status st = check_solver(h);
    if (st) return st;
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    h->stream = (cudaStream_t)cuda_stream; /* NULL: the legacy default stream */
    return BES_OK;
}

bes_status bes_last_solve_ms(bes_solver* h, float* ms) {
    bes_status st = check_solver(h);
    if (st) return st;
    if (!ms) return BES_ERR_ARGUMENT;
    CUDA_TRY(h, cudaEventSynchronize(h->t1));
    CUDA_TRY(h, cudaEventElapsedTime(ms, h->t0, h->t1));
    return BES_OK;
}

bes_status bes_last_solve_launches(bes_solver* h, int32_t* launches) {
    if (!h || !launches) return BES_ERR_ARGUMENT;
    *launches = h->last_launches;
    return BES_OK;
}

bes_status bes_get_counters(bes_solver* h, int32_t sid, bes_counters* out) {
    if (!h || !out) return BES_ERR_ARGUMENT;
    bes_status st = bound(h, "bes_get_counters", "SystemNumber", sid, 0, h->n_systems - 1);
    if (st) return st;
    out->accepted_steps = ((uint64_t*)h->buf[B_CNT_ACC].h)[sid];
    out->rejected_steps = ((uint64_t*)h->buf[B_CNT_REJ].h)[sid];
    out->bicg_iterations = ((uint64_t*)h->buf[B_CNT_BICG].h)[sid];
    out->rhs_evaluations = ((uint64_t*)h->buf[B_CNT_RHS].h)[sid];
    out->status = ((int32_t*)h->buf[B_STATUS].h)[sid];
    out->units = h->units[sid];
    return BES_OK;
}

bes_status bes_reset_counters(bes_solver* h) {
    bes_status st = check_solver(h);
    if (st) return st;
    const int ids[] = {B_CNT_ACC, B_CNT_REJ, B_CNT_BICG, B_CNT_RHS, B_STATUS};
    for (int id : ids) {
        Buf& b = h->buf[id];
        CUDA_TRY(h, cudaMemsetAsync(b.d, 0, b.bytes(), h->stream));
        std::memset(b.h, 0, b.bytes());
    }
    return BES_OK;
}

/* ---------------- text inputs ---------------- */

static bes_status read_numbers(const char* fn, const char* path, int64_t n, double* out) {
    if (!path || !out || n < 0) return fail(nullptr, BES_ERR_ARGUMENT, "%s: bad argument", fn);
    FILE* f = std::fopen(path, "r");
    if (!f) return fail(nullptr, BES_ERR_IO, "%s: cannot open '%s': %s", fn, path, std::strerror(errno));
    for (int64_t i = 0; i < n; i++) {
        double v;
        if (std::fscanf(f, "%lf", &v) != 1) {
            std::fclose(f);
            return fail(nullptr, BES_ERR_IO, "%s: '%s' holds fewer than %lld numbers (stopped at %lld)", fn, path,
                        (long long)n, (long long)i);
        }
        out[i] = v;
    }
    std::fclose(f);
    return BES_OK;
}

bes_status bes_load_bubble_sizes(const char* path, int32_t n, double* out) {
    return read_numbers("bes_load_bubble_sizes", path, n, out);
}

bes_status bes_load_coupling_matrix(const char* path, int32_t n, double* out) {
    return read_numbers("bes_load_coupling_matrix", path, (int64_t)n * n, out);
}

}  // extern "C"
