/*
 * bes_oracle.h -- TEST INFRASTRUCTURE.  The CPU oracle for the coupled
 * Keller-Miksis ensemble integrator.  Only the tests, the smoke check and the
 * CPU-baseline leg of the benchmark load it; the product never does.
 *
 * It restates, in plain C++ FP64, the reference's per-block solver for one
 * system at a time (the reference has no CPU path):
 *   step loop          SourceCodes/CoupledSystmes_PerBlock_Solver.cuh:329-572
 *   RKCK45 stepper     SourceCodes/CoupledSystems_PerBlock_ExplicitRungeKutta_Steppers.cuh:94-425
 *   BiCG coupling solve   ...ExplicitRungeKutta_Steppers.cuh:432-562 (helpers :565-805)
 *   error controller   SourceCodes/CoupledSystems_PerBlock_ExplicitRungeKutta_ErrorControllers.cuh:454-542
 *   RK4 controller     ...ExplicitRungeKutta_ErrorControllers.cuh:424-450
 *   event step control SourceCodes/CoupledSystems_PerBlock_EventHandling.cuh:216-268
 *   dense output       SourceCodes/CoupledSystems_PerBlock_DenseOutput.cuh:312-395
 *   Keller-Miksis model and collapse callbacks  BubbleEnsemble_SystemDefinition.cuh:8-126
 *   per-period driver semantics (Solve() = one period, accessory reset)
 *                      CollapseStrength.cu:122-147, SourceCodes/CoupledSystems_PerBlock_Interface.cuh:1951-1956
 *
 * Arrays use the canonical structure-of-arrays layout of the product's C ABI:
 * unit-scope component k of unit u of system s lives at
 * [k * total_units + unit_offset[s] + u]; system-scope component k of system
 * s at [k * n_systems + s].
 */
#ifndef BES_ORACLE_H
#define BES_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BES_ORACLE_UD 2
#define BES_ORACLE_NUP 21
#define BES_ORACLE_NCOLL 32
#define BES_ORACLE_NUA (2 * BES_ORACLE_NCOLL)
#define BES_ORACLE_NIUA 1
#define BES_ORACLE_NE 1

/* status bits per system (same meaning as the product's) */
#define BES_ORACLE_ST_NONFINITE 1       /* terminated: non-finite state at the minimum step */
#define BES_ORACLE_ST_MIN_STEP 2        /* a step was forced through at the minimum step size */
#define BES_ORACLE_ST_STEP_BUDGET 4     /* the per-period step budget ran out */
#define BES_ORACLE_ST_EVENT_MISSED 8    /* an event cut would have gone below the minimum step */
#define BES_ORACLE_ST_BICG_CAP 16       /* a BiCG solve used every iteration without meeting its exit test */

typedef struct bes_oracle_problem {
    int32_t n_systems;
    int32_t active_systems;
    int64_t total_units;
    const int32_t* units;            /* [n_systems] */
    const int64_t* unit_offset;      /* [n_systems] */
    const int64_t* coupling_offset;  /* [n_systems], in doubles, into `coupling` */
    const double* coupling;          /* N x N column-major matrices */
    double* state;                   /* [UD][total_units] */
    const double* upar;              /* [NUP][total_units] */
    double* uacc;                    /* [NUA][total_units] */
    int32_t* iuacc;                  /* [NIUA][total_units] */
    double* time_domain;             /* [2][n_systems] */
    double* actual_time;             /* [n_systems] */
    const double* rtol;              /* [UD][n_systems] */
    const double* atol;              /* [UD][n_systems] */
    double event_tol;
    int32_t event_dir;
    int32_t algorithm;               /* 0 = RK4, 1 = RKCK45 */
    double dt0, dtmin, dtmax, grow, shrink;
    int32_t bicg_max_iter;           /* the reference's loop runs iter = 1..19 */
    int32_t shared_assoc;            /* 1: systems with N > 32 use the shared-matrix association (see .cpp) */
    int64_t max_steps_per_period;    /* attempted steps per period before STEP_BUDGET */
    int32_t ndo;                     /* dense output slots per system */
    int32_t do_save_frequency;
    double do_min_dt;
    double* dense_time;              /* [ndo][n_systems] */
    double* dense_state;             /* [ndo][UD][total_units] */
    int32_t* dense_index;            /* [n_systems] */
    /* outputs, accumulated: [n_systems] */
    int64_t* n_accepted;
    int64_t* n_rejected;
    int64_t* n_bicg_iter;
    int64_t* n_rhs;
    int32_t* status;
    /* coupling factors of the shared-matrix association, [total_units] each, or NULL (= 1):
     * system s couples units i, j through a_i G_ij b_j, G its stored matrix */
    const double* coupling_row_scale;
    const double* coupling_col_scale;
    /* 0: the reference's BiCG recurrence (two reductions per iteration);
     * 1: the single-reduction recurrence (see coupled_rhs in the .cpp) */
    int32_t bicg_variant;
    int32_t pad;
    /* optional [n_systems] output, or NULL: the smallest step size attempted
     * (min over the periods of this call and the value already stored) */
    double* min_dt;
    /* > 0: the coupling matrices are banded (2 band_width + 1 wrapping
     * diagonals, the reference's CBW storage) and systems with
     * 2 band_width + 1 < N use the banded association (see coupled_rhs) */
    int32_t band_width;
    int32_t pad2;
} bes_oracle_problem;

/* Integrate `n_periods` reference Solve() calls for every active system.
 * Before period index `reset_at` (if 0 <= reset_at < n_periods) every unit's
 * accessories are set to uacc_reset[k] / iuacc_reset[k].
 * n_threads <= 0 uses all OpenMP threads.  Returns 0 on success. */
int bes_oracle_solve(const bes_oracle_problem* p, int n_periods, int reset_at,
                     const double* uacc_reset, const int32_t* iuacc_reset, int n_threads);

/* Elementary functions of the oracle (for the accuracy tests). */
double bes_oracle_pow(double x, double y);
double bes_oracle_pow_recip(double x, double y);   /* (1/x)^y */
double bes_oracle_exp(double x);
double bes_oracle_log(double x);
void bes_oracle_sincospi(double x, double* s, double* c);
void bes_oracle_sincos(double x, double* s, double* c);

/* One coupled right-hand side of a whole system (tests of the BiCG solve):
 * state [2][n] (SoA), upar [21][n], coupling n x n column-major.
 * Writes f [2][n] and returns the number of completed BiCG iterations. */
int bes_oracle_rhs(int n, double t, const double* state, const double* upar,
                   const double* coupling, int bicg_max_iter, double* f);

int bes_oracle_max_threads(void);

/* number of single-reduction BiCG solves redone with the reference's
 * recurrence since the last reset (reset != 0 clears it) */
long long bes_oracle_rec1_fallbacks(int reset);
/* of those, the solves the iteration cap ended */
long long bes_oracle_rec1_fallbacks_capped(int reset);

#ifdef __cplusplus
}
#endif

#endif
