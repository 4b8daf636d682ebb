/*
 * bes.h -- C ABI of the B200 ensemble integrator for coupled Keller-Miksis
 * bubble systems ("bes" = bubble ensemble solver).
 *
 * This is the drop-in boundary for the reference's host API, the compile-time
 * C++ class ProblemSolver<NS,UPS,UD,TPB,SPB,NC,CBW,CCI,NUP,NSP,NGP,NiGP,NUA,
 * NiUA,NSA,NiSA,NE,NDO,Algorithm,Precision>
 * (SourceCodes/CoupledSystems_PerBlock_Interface.cuh:135-248).  Each entry
 * point below names the member function it replaces.  Plain C types only: a
 * ctypes / cgo / JNI binding needs nothing else.  include/bes_problem_solver.h
 * rebuilds the reference's template class on top of these calls.
 *
 * Differences from the reference, by design:
 *   - sizes are run-time values (bes_config) and unit counts may differ per
 *     system; the system definition (the seven device callbacks and their
 *     sizes) is compiled into the library, and bes_create checks the sizes;
 *   - every call returns a bes_status instead of calling exit() (the
 *     reference exits on bad indices, Interface.cuh:718-733, and on CUDA
 *     errors, :13-22); bes_last_error() gives the message;
 *   - bes_solve_periods() runs many Solve() periods, with the accessory reset
 *     between the transient and the recorded phase, in one kernel launch;
 *   - per-system status and counters (steps, rejections, BiCG iterations)
 *     are returned to the host.
 * A handle is not thread-safe; separate handles are independent.
 */
#ifndef BES_H
#define BES_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t bes_status;
#define BES_OK 0
#define BES_ERR_ARGUMENT 1      /* null pointer, bad size or value */
#define BES_ERR_INDEX 2         /* index out of range (reference: BoundCheck, Interface.cuh:718-733) */
#define BES_ERR_OPTION 3        /* option/variable not valid for this call (reference: exit in the switch defaults) */
#define BES_ERR_CUDA 4          /* CUDA runtime error (reference: gpuErrCHK, Interface.cuh:13-22) */
#define BES_ERR_MEMORY 5        /* allocation failed or too large (reference: Interface.cuh:463-471) */
#define BES_ERR_IO 6            /* input file missing or malformed */
#define BES_ERR_MODEL 7         /* sizes do not match the compiled system definition */
#define BES_ERR_UNSUPPORTED 8   /* feature outside this build (e.g. banded coupling storage) */

/* ListOfVariables, same names and order as Interface.cuh:35-53 */
#define BES_ALL 0
#define BES_TIME_DOMAIN 1
#define BES_ACTUAL_TIME 2
#define BES_ACTUAL_STATE 3
#define BES_UNIT_PARAMETERS 4
#define BES_SYSTEM_PARAMETERS 5
#define BES_GLOBAL_PARAMETERS 6
#define BES_INTEGER_GLOBAL_PARAMETERS 7
#define BES_UNIT_ACCESSORIES 8
#define BES_INTEGER_UNIT_ACCESSORIES 9
#define BES_SYSTEM_ACCESSORIES 10
#define BES_INTEGER_SYSTEM_ACCESSORIES 11
#define BES_COUPLING_MATRIX 12
#define BES_COUPLING_STRENGTH 13
#define BES_COUPLING_INDEX 14
#define BES_DENSE_OUTPUT 15
#define BES_DENSE_INDEX 16
#define BES_DENSE_TIME 17
#define BES_DENSE_STATE 18
/* extensions (no reference counterpart) */
#define BES_RELATIVE_TOLERANCE_SYSTEM 100  /* [UD][n_systems] per-system relative tolerances */
#define BES_ABSOLUTE_TOLERANCE_SYSTEM 101  /* [UD][n_systems] per-system absolute tolerances */
#define BES_COUNTERS 102                   /* per-system counters and status (device -> host only) */
#define BES_COUPLING_ROW_SCALE 103         /* [total_units] a_i and                                        */
#define BES_COUPLING_COLUMN_SCALE 104      /* [total_units] b_j of a system's coupling matrix
                                              C_ij = a_i G_ij b_j, G the stored (shared) matrix; default 1.
                                              One geometry G = 1/d_ij serves systems with their own radii
                                              (a_i = R_i^-2, b_j = R_j^3).  Applied by the shared-matrix
                                              kernels only (SharedCouplingMatrices, more than 32 units);
                                              a solve with other launches and factors != 1 is an error. */
#define BES_POINCARE_SECTIONS 105          /* [sections][total_units] per-period analysis outputs (device -> host), */
#define BES_PERIOD_NUMBER 106              /* [total_units] int32       see bes_set_period_analysis              */
#define BES_MAXIMUM_ACCESSORY 107          /* [total_units]                                                       */

/* ListOfSolverOptions, same names and order as Interface.cuh:55-68 */
#define BES_OPT_INITIAL_TIME_STEP 0
#define BES_OPT_ACTIVE_SYSTEMS 1
#define BES_OPT_MAXIMUM_TIME_STEP 2
#define BES_OPT_MINIMUM_TIME_STEP 3
#define BES_OPT_TIME_STEP_GROW_LIMIT 4
#define BES_OPT_TIME_STEP_SHRINK_LIMIT 5
#define BES_OPT_RELATIVE_TOLERANCE 6
#define BES_OPT_ABSOLUTE_TOLERANCE 7
#define BES_OPT_EVENT_TOLERANCE 8
#define BES_OPT_EVENT_DIRECTION 9
#define BES_OPT_DENSE_OUTPUT_SAVE_FREQUENCY 10
#define BES_OPT_DENSE_OUTPUT_MINIMUM_TIME_STEP 11
#define BES_OPT_SHARED_GLOBAL_VARIABLES 12
#define BES_OPT_SHARED_COUPLING_MATRICES 13
/* extensions */
#define BES_OPT_MAX_STEPS_PER_PERIOD 100   /* attempted steps per period before BES_STATUS_STEP_BUDGET (default 1e6) */
#define BES_OPT_BICG_MAX_ITERATIONS 101    /* the reference's loop runs 19 iterations (Steppers.cuh:508) */
#define BES_OPT_WARPS_PER_BLOCK 102        /* launch shape: systems (warps) per CTA, 0 = automatic */
#define BES_OPT_USE_CUDA_GRAPH 103         /* 1 (default): bes_solve_periods captures its launches once into a
                                              CUDA graph and replays it; 0: direct launches */
#define BES_OPT_WARPS_PER_SYSTEM 104       /* 0 (default): systems of 33-64 units run on 2 warps and of 65-128
                                              units on 4 warps (one unit per lane); 1: one warp per system
                                              (2 or 4 units per lane).  Results are bit-identical. */
#define BES_OPT_BICG_RECURRENCE 105        /* 0 (default): the reference's BiCG recurrence (Steppers.cuh:508-561:
                                              two reductions per iteration); 1: the single-reduction form of the
                                              same iterates (residual products first, rho = r.r~ and mu = r~.Ar
                                              in one reduction, sigma = mu - beta^2 sigma_prev).  A solve of form
                                              1 stands only if x is finite and the true residual b - A x passes
                                              the reference's exit test; otherwise (and at the iteration cap) it
                                              is redone with form 0.  Equal in exact arithmetic, rounded
                                              differently: results stay within the parity tolerances of the
                                              reference, not bit-identical to option 0. */

/* Algorithms, Interface.cuh:33 */
#define BES_RK4 0
#define BES_RKCK45 1

/* per-system status bits (the reference only printf()s these) */
#define BES_STATUS_NONFINITE 1
#define BES_STATUS_MIN_STEP 2
#define BES_STATUS_STEP_BUDGET 4
#define BES_STATUS_EVENT_MISSED 8
#define BES_STATUS_BICG_CAP 16

typedef struct bes_solver bes_solver;

/* Problem sizes: the reference's template parameters
 * (CollapseStrength.cu:34-54), as run-time values. */
typedef struct bes_config {
    int32_t device;
    int32_t n_systems;                 /* NS */
    int32_t units_per_system;          /* UPS for uniform ensembles; 0 when `units` is given */
    const int32_t* units;              /* optional [n_systems] unit count per system (1..128) */
    int32_t unit_dim;                  /* UD */
    int32_t n_unit_parameters;         /* NUP */
    int32_t n_system_parameters;       /* NSP */
    int32_t n_global_parameters;       /* NGP */
    int32_t n_int_global_parameters;   /* NiGP */
    int32_t n_unit_accessories;        /* NUA */
    int32_t n_int_unit_accessories;    /* NiUA */
    int32_t n_system_accessories;      /* NSA */
    int32_t n_int_system_accessories;  /* NiSA */
    int32_t n_events;                  /* NE */
    int32_t n_dense_output;            /* NDO */
    int32_t n_couplings;               /* NC; coupling 0 enters the implicit solve (as in the reference) */
    int32_t coupling_bandwidth;        /* CBW: 0 full storage, > 0 a (wrapping) band of 2 CBW + 1 diagonals */
    int32_t coupling_circular;         /* CCI: 1 one value per diagonal for every row (circulant); see
                                          bes_set_host_coupling */
    int32_t algorithm;                 /* BES_RK4 or BES_RKCK45 */
    int32_t n_coupling_matrices;       /* distinct geometries; 1 = one matrix for every system (the reference) */
    const int32_t* coupling_matrix_of_system; /* optional [n_systems]; default s -> 0, or s -> s when
                                                 n_coupling_matrices == n_systems */
} bes_config;

/* sizes of the system definition compiled into the library */
typedef struct bes_model_info {
    int32_t unit_dim, n_unit_parameters, n_system_parameters, n_global_parameters, n_int_global_parameters;
    int32_t n_unit_accessories, n_int_unit_accessories, n_system_accessories, n_int_system_accessories;
    int32_t n_events;
    int32_t max_units_per_system;
    char name[64];
} bes_model_info;

typedef struct bes_counters {
    uint64_t accepted_steps;
    uint64_t rejected_steps;
    uint64_t bicg_iterations;          /* completed BiCG iterations summed over all right-hand sides */
    uint64_t rhs_evaluations;
    int32_t status;                    /* OR of BES_STATUS_* */
    int32_t units;
} bes_counters;

/* ProblemSolver::ProblemSolver(int Device), Interface.cuh:354-657: allocates
 * pinned host mirrors and device arrays, sets the default options
 * (Interface.cuh:613-635). */
bes_status bes_create(const bes_config* config, bes_solver** out);
/* ProblemSolver::~ProblemSolver, Interface.cuh:661-714 */
bes_status bes_destroy(bes_solver* h);
/* sizes of the compiled system definition (BubbleEnsemble_SystemDefinition.cuh) */
bes_status bes_model_info_get(bes_model_info* out);

/* ProblemSolver::SolverOption(ListOfSolverOptions, T), Interface.cuh:774-827 */
bes_status bes_solver_option(bes_solver* h, int32_t option, double value);
/* ProblemSolver::SolverOption(ListOfSolverOptions, int, T), Interface.cuh:832-865 */
bes_status bes_solver_option_indexed(bes_solver* h, int32_t option, int32_t index, double value);

/* ProblemSolver::SetHost overloads (SourceCodes/CoupledSystems_PerBlock_Interface.cuh):
 * unit scope :870-910, system scope and dense time :914-965, global scope :969-997,
 * coupling matrix :1001-1087, dense index :1091-1110, dense state :1114-1140.
 * With several coupling matrices, `n` = matrix * n_couplings + coupling. */
bes_status bes_set_host_unit(bes_solver* h, int32_t sid, int32_t uid, int32_t var, int32_t k, double value);
bes_status bes_set_host_system(bes_solver* h, int32_t sid, int32_t var, int32_t k, double value);
bes_status bes_set_host_global(bes_solver* h, int32_t var, int32_t k, double value);
bes_status bes_set_host_coupling(bes_solver* h, int32_t n, int32_t var, int32_t row, int32_t col, double value);
bes_status bes_set_host_dense_index(bes_solver* h, int32_t sid, int32_t var, double value);
bes_status bes_set_host_dense_state(bes_solver* h, int32_t sid, int32_t uid, int32_t var, int32_t comp,
                                    int32_t slot, double value);
/* ProblemSolver::GetHost overloads: unit :1341-1377, system and dense time :1381-1425,
 * global :1429-1454, coupling matrix :1458-1478, dense index :1482-1500, dense state :1504-1529 */
bes_status bes_get_host_unit(bes_solver* h, int32_t sid, int32_t uid, int32_t var, int32_t k, double* value);
bes_status bes_get_host_system(bes_solver* h, int32_t sid, int32_t var, int32_t k, double* value);
bes_status bes_get_host_global(bes_solver* h, int32_t var, int32_t k, double* value);
bes_status bes_get_host_coupling(bes_solver* h, int32_t n, int32_t var, int32_t row, int32_t col, double* value);
bes_status bes_get_host_dense_index(bes_solver* h, int32_t sid, int32_t var, double* value);
bes_status bes_get_host_dense_state(bes_solver* h, int32_t sid, int32_t uid, int32_t var, int32_t comp,
                                    int32_t slot, double* value);

/* Bulk copy between a caller array and the host mirror, in the canonical
 * layout (unit scope [k][total_units], system scope [k][n_systems], coupling
 * matrices back to back, column-major).  `count` is in elements; integer
 * variables take int32_t, the rest double.  No reference counterpart (the
 * reference only has element-wise SetHost/GetHost). */
bes_status bes_set_array(bes_solver* h, int32_t var, const void* src, int64_t count);
bes_status bes_get_array(bes_solver* h, int32_t var, void* dst, int64_t count);
bes_status bes_array_size(bes_solver* h, int32_t var, int64_t* count);

/* ProblemSolver::SynchroniseFromHostToDevice, Interface.cuh:1144-1238, and
 * SynchroniseFromDeviceToHost, Interface.cuh:1242-1336
 * (asynchronous on the solver's stream, like the reference) */
bes_status bes_synchronise_host_to_device(bes_solver* h, int32_t var);
bes_status bes_synchronise_device_to_host(bes_solver* h, int32_t var);

/* ProblemSolver::Solve, Interface.cuh:1951-1956: one period (one kernel launch),
 * asynchronous. */
bes_status bes_solve(bes_solver* h);
/* The driver loop of CollapseStrength.cu:123-147 (n Solve() calls, accessories
 * reset before period `reset_at`, -1 for never) in one persistent launch. */
bes_status bes_solve_periods(bes_solver* h, int32_t n_periods, int32_t reset_at);
/* reset values for bes_solve_periods (CollapseStrength.cu:373-396 resets every
 * unit's accessories to 0 and its integer accessory to -1) */
bes_status bes_set_accessory_reset(bes_solver* h, const double* uacc, const int32_t* iuacc);

/* ProblemSolver::SynchroniseDevice / InsertSynchronisationPoint / SynchroniseSolver,
 * Interface.cuh:1960-1983 */
bes_status bes_synchronise_device(bes_solver* h);
bes_status bes_insert_synchronisation_point(bes_solver* h);
bes_status bes_synchronise_solver(bes_solver* h);

/* Use the caller's CUDA stream (a cudaStream_t; NULL is the legacy default
 * stream) instead of the solver's own stream for every later call. */
bes_status bes_set_stream(bes_solver* h, void* cuda_stream);
/* device time of the last bes_solve / bes_solve_periods, measured with CUDA
 * events around its launches (valid after bes_synchronise_solver) */
bes_status bes_last_solve_ms(bes_solver* h, float* ms);
/* number of kernel launches the last bes_solve / bes_solve_periods issued */
bes_status bes_last_solve_launches(bes_solver* h, int32_t* launches);

/* per-system counters from the host mirror; call
 * bes_synchronise_device_to_host(h, BES_COUNTERS) and sync first */
bes_status bes_get_counters(bes_solver* h, int32_t sid, bes_counters* out);
/* zero the device counters and status words */
bes_status bes_reset_counters(bes_solver* h);

/* LoadBubbleSizes, CollapseStrength.cu:245-258: n whitespace-separated numbers */
bes_status bes_load_bubble_sizes(const char* path, int32_t n, double* out);
/* LoadCouplingMatrix, CollapseStrength.cu:260-277: n x n numbers, row by row,
 * written to out[row * n + col] */
bes_status bes_load_coupling_matrix(const char* path, int32_t n, double* out);

/* ListCUDADevices, Interface.cuh:260-296 */
bes_status bes_device_count(int32_t* count);

typedef struct bes_device_info {
    char name[256];
    int32_t cc_major, cc_minor;
    int32_t multiprocessors;
    int32_t pad;
    uint64_t global_memory_bytes;
} bes_device_info;
/* PrintPropertiesOfSpecificDevice / SelectDeviceByClosestRevision, Interface.cuh:298-346 */
bes_status bes_device_info_get(int32_t device, bes_device_info* out);

/* Utility, no reference counterpart: the device's FP64 fused multiply-add
 * throughput in TFLOP/s (2 flops per FMA), measured with an FMA loop that
 * keeps 8 independent chains per thread on every SM; the roofline
 * denominator of the FP64 solver kernel. */
bes_status bes_measure_fp64_peak(int32_t device, double* tflops);

/* ---- per-period analysis on the device (BubbleEnsemble.cu:174-216 runs it on
 * the host after every Solve()) ----
 * sections >= 0 turns it on for the following bes_solve_periods calls: each
 * call takes every unit's state at its start as the reference point, stores
 * state component 0 after each of its first `sections` periods
 * (BES_POINCARE_SECTIONS, [sections][total_units]), records the first period
 * (1-based) whose end state lies within distance_tolerance of the reference
 * point (Euclidean over the state components; BES_PERIOD_NUMBER, int32
 * [total_units], 0: none) and the running maximum over period ends of unit
 * accessory accessory_index, starting from its value at the call's start
 * (BES_MAXIMUM_ACCESSORY, [total_units]).  The reference uses tolerance 1e-6
 * and accessory 0.  sections < 0 turns it off and frees the arrays. */
bes_status bes_set_period_analysis(bes_solver* h, int32_t sections, double distance_tolerance,
                                   int32_t accessory_index);
/* Print(var) and Print(var, n) of ProblemSolver (Interface.cuh:1809-1947):
 * the host mirror of `var` to <Name>InSolverObject.txt in `directory` (NULL:
 * the working directory) in the reference's layout and number format;
 * serial selects the matrix (BES_COUPLING_MATRIX) or the system
 * (BES_DENSE_OUTPUT: DenseOutput_<serial>.txt) and is ignored otherwise. */
bes_status bes_print(bes_solver* h, int32_t var, int32_t serial, const char* directory);
/* Output files of the reference drivers (CollapseStrength.cu:174-198,
 * BubbleEnsemble.cu:435-491) from the host mirrors, same layout and number
 * formats; kind is one of BES_CSV_*. */
#define BES_CSV_COLLAPSE 0
#define BES_CSV_POINCARE 1
#define BES_CSV_PERIOD 2
#define BES_CSV_EXPANSION 3
bes_status bes_write_csv(bes_solver* h, int32_t kind, const char* path);

/* ---- launch-shape autotuner (no reference counterpart; the reference fixes
 * threads and systems per block at compile time, Interface.cuh:135-248) ----
 * Times every launch shape of every non-empty size class on the device's
 * current inputs (n_periods periods, each system's attempted steps capped at
 * step_cap per period when step_cap > 0), keeps the fastest per class for the
 * following solves and restores the device state it started from.  Shapes
 * give bit-identical results.  Setting BES_OPT_WARPS_PER_BLOCK or
 * BES_OPT_WARPS_PER_SYSTEM afterwards replaces the tuned choice. */
typedef struct bes_autotune_result {
    int32_t warps_per_block[3];    /* per size class (N <= 32, <= 64, <= 128); 0 where the class is empty */
    int32_t warps_per_system[3];   /* 0: 2 or 4 warps per system above 32 units, 1: one warp */
    float ms[3];                   /* device time of the chosen shape */
    int32_t candidates;            /* shapes timed in all */
} bes_autotune_result;
bes_status bes_autotune(bes_solver* h, int32_t n_periods, int64_t step_cap, bes_autotune_result* result);

/* No counterpart in the reference.  For callers that cannot allocate device
 * memory: an application that already owns the GPU's memory (a framework that
 * reserves the device and hands out slices of its own pool, or a real-time
 * loop in which cudaMalloc could block or synchronise) lays out every input
 * and output in memory it holds and passes device pointers here; the call
 * allocates nothing (no cudaMalloc, no cudaFree, no host allocation).
 * Arrays use the layout of bes_get_array / bes_set_array for the compiled
 * system definition (bes_model_info_get).  The solver's scratch (per-class
 * work counters and the processing order) is a fixed device array inside the
 * library, held by every GPU that loads it until exit: at most
 * BES_NOALLOC_MAX_SYSTEMS systems per call; larger ensembles are rejected
 * with BES_ERR_ARGUMENT.  The first call on a device (with that device
 * current) looks up the scratch's device address; make that first call before
 * any stream capture.  Every call resets the scratch before its launches, and
 * all calls share it: calls that overlap on the GPU race and must be
 * serialised by the caller.  Runs asynchronously on `stream` (NULL: the
 * legacy default stream) and integrates n_periods periods of systems
 * [0, n_systems), resetting accessories before period reset_at, like
 * bes_solve_periods. */
#define BES_NOALLOC_MAX_SYSTEMS 65536
typedef struct bes_noalloc_problem {
    int32_t n_systems;
    int32_t algorithm;                 /* BES_RK4 or BES_RKCK45 */
    int64_t total_units;
    const int32_t* units_host;         /* host copy of the unit counts [n_systems] (launch planning); must
                                          hold the same values as the device array `units` (a system whose
                                          class disagrees may be skipped, never read out of bounds) */
    /* device arrays */
    const int32_t* units;              /* [n_systems] */
    const int64_t* unit_offset;        /* [n_systems] */
    const int64_t* coupling_offset;    /* [n_systems], in doubles */
    const double* coupling;            /* N x N column-major matrices */
    double* state;                     /* [UD][total_units] */
    const double* upar;                /* [NUP][total_units] */
    double* uacc;                      /* [NUA][total_units] */
    int32_t* iuacc;                    /* [NiUA][total_units] */
    double* spar;                      /* [NSP][n_systems] (may be NULL when NSP = 0) */
    double* sacc;                      /* [NSA][n_systems] */
    int32_t* isacc;                    /* [NiSA][n_systems] */
    double* gpar;                      /* [NGP] */
    int32_t* igpar;                    /* [NiGP] */
    double* time_domain;               /* [2][n_systems] */
    double* actual_time;               /* [n_systems] */
    const double* rtol;                /* [UD][n_systems] */
    const double* atol;                /* [UD][n_systems] */
    const double* event_tol;           /* [NE] */
    const int32_t* event_dir;          /* [NE] */
    const double* uacc_reset;          /* [NUA] */
    const int32_t* iuacc_reset;        /* [NiUA] */
    double* dense_time;                /* [ndo][n_systems] (NULL when ndo = 0) */
    double* dense_state;               /* [ndo][UD][total_units] */
    int32_t* dense_index;              /* [n_systems] */
    uint64_t* n_accepted;              /* [n_systems] counters, accumulated */
    uint64_t* n_rejected;
    uint64_t* n_bicg_iter;
    uint64_t* n_rhs;
    int32_t* status;                   /* [n_systems], OR of BES_STATUS_* */
    /* options: a field left 0 takes the default of SolverOption (Interface.cuh:613-618):
     * dt0 1e-2, dtmin 1e-12, dtmax 1e6, grow 5, shrink 0.1, bicg_max_iter 19,
     * max_steps_per_period 1e6, do_save_frequency 1 (do_min_dt and ndo: 0);
     * a negative dt0, dtmin, dtmax, grow or shrink is rejected with BES_ERR_ARGUMENT */
    double dt0, dtmin, dtmax, grow, shrink, do_min_dt;
    int32_t ndo, do_save_frequency;
    int32_t bicg_max_iter, warps_per_block;
    int64_t max_steps_per_period;
    char* error_message;               /* optional caller buffer for a message on failure */
    int32_t error_capacity;
    int32_t bicg_recurrence;           /* BES_OPT_BICG_RECURRENCE: 0 (reference) or 1 */
} bes_noalloc_problem;
bes_status bes_solve_periods_noalloc(const bes_noalloc_problem* problem, int32_t n_periods, int32_t reset_at,
                                     void* stream);

/* ---- surrogate network (no reference counterpart) -------------------------
 * A small MLP (n_in -> width x depth (GELU) -> n_out) trained and evaluated
 * by the library's own CUDA kernels: BF16 weights and activations, FP32
 * master weights, FP32 accumulation, Adam.  It maps sweep parameters
 * (amplitude, frequency, radius statistics) to collapse outputs so that a
 * sweep integrates only the points it flags.  x, y, target are device
 * pointers to row-major [batch][n] FP32 arrays. */
typedef struct bes_mlp bes_mlp;
typedef struct bes_mlp_config {
    int32_t device;
    int32_t n_in, width, depth, n_out;
    int32_t max_batch;
    uint64_t seed;
} bes_mlp_config;
bes_status bes_mlp_create(const bes_mlp_config* config, bes_mlp** out);
bes_status bes_mlp_destroy(bes_mlp* m);
bes_status bes_mlp_parameter_count(bes_mlp* m, int64_t* count);
/* standardisation of inputs and targets (host arrays) */
bes_status bes_mlp_set_normalization(bes_mlp* m, const float* in_mean, const float* in_std, const float* out_mean,
                                     const float* out_std);
bes_status bes_mlp_get_parameters(bes_mlp* m, float* host, int64_t count);
bes_status bes_mlp_set_parameters(bes_mlp* m, const float* host, int64_t count);
bes_status bes_mlp_get_gradients(bes_mlp* m, float* host, int64_t count);
bes_status bes_mlp_forward(bes_mlp* m, const float* x, int32_t batch, float* y, void* stream);
/* gradients of the mean squared error of the standardised outputs; loss (host) optional */
bes_status bes_mlp_backward(bes_mlp* m, const float* x, const float* target, int32_t batch, float* loss,
                            void* stream);
bes_status bes_mlp_adam_step(bes_mlp* m, float learning_rate, void* stream);
const char* bes_mlp_last_error(const bes_mlp* m);

const char* bes_status_string(bes_status status);
const char* bes_last_error(const bes_solver* h);

#ifdef __cplusplus
}
#endif

#endif
