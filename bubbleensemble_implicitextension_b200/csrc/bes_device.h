/*
 * bes_device.h -- the solver kernel's argument block (host and device view).
 *
 * HBM layout (all arrays device-resident, structure of arrays):
 *   unit scope   component k of unit u of system s at [k*total_units + unit_offset[s] + u]
 *                (state, unit parameters, unit accessories, dense states per slot);
 *   system scope component k of system s at [k*n_systems + s]
 *                (time domain, actual time, tolerances, system parameters/accessories);
 *   coupling     one N x N column-major matrix per distinct geometry, system s uses the
 *                matrix at coupling_offset[s] (systems may share one matrix); with the
 *                shared-matrix kernels the matrix of unit pair (i, j) is a_i G_ij b_j,
 *                a and b unit-scope factors (1 unless set).
 * This is the reference's layout (SourceCodes/CoupledSystems_PerBlock_Interface.cuh:875-879,
 * :918-919, :1007, :1124-1125) with the per-block thread padding removed and ragged
 * unit counts allowed.
 */
#ifndef BES_DEVICE_H
#define BES_DEVICE_H

#include <stdint.h>

namespace bes {

struct DeviceProblem {
    int32_t n_systems;
    int32_t n_active;                /* systems [0, n_active) are integrated */
    int64_t total_units;
    const int32_t* units;            /* [n_systems] */
    const int64_t* unit_offset;      /* [n_systems] */
    const int64_t* coupling_offset;  /* [n_systems] offset (doubles) of the system's matrix */
    const double* coupling;
    const double* coupling_row_scale;  /* [total_units] a_i, or NULL: the shared-matrix kernels use  */
    const double* coupling_col_scale;  /* [total_units] b_j    C_ij = a_i G_ij b_j with G the stored matrix */
    const int32_t* order;            /* [n_active] processing order (costliest first) */
    double* state;                   /* [UD][total_units] */
    const double* upar;              /* [NUP][total_units] */
    double* uacc;                    /* [NUA][total_units] */
    int32_t* iuacc;                  /* [NIUA][total_units] */
    double* spar;                    /* [NSP][n_systems] */
    double* sacc;                    /* [NSA][n_systems] */
    int32_t* isacc;                  /* [NISA][n_systems] */
    double* gpar;                    /* [NGP] */
    int32_t* igpar;                  /* [NIGP] */
    double* time_domain;             /* [2][n_systems] */
    double* actual_time;             /* [n_systems] */
    const double* rtol;              /* [UD][n_systems] */
    const double* atol;              /* [UD][n_systems] */
    const double* event_tol;         /* [NE] */
    const int32_t* event_dir;        /* [NE] */
    double dt0, dtmin, dtmax, grow, shrink;
    int32_t algorithm;               /* 0 RK4, 1 RKCK45 */
    int32_t bicg_max_iter;
    int64_t max_steps_per_period;
    int32_t ndo, do_save_frequency;
    double do_min_dt;
    double* dense_time;              /* [ndo][n_systems] */
    double* dense_state;             /* [ndo][UD][total_units] */
    int32_t* dense_index;            /* [n_systems] */
    unsigned long long* n_accepted;  /* [n_systems], accumulated */
    unsigned long long* n_rejected;
    unsigned long long* n_bicg_iter;
    unsigned long long* n_rhs;
    int32_t* status;                 /* [n_systems], OR of BES_STATUS_* bits */
    int32_t* work_counter;           /* one int, zeroed before each launch */
    int32_t n_periods;
    int32_t reset_at;                /* period index before which accessories are reset (-1: never) */
    const double* uacc_reset;        /* [NUA] */
    const int32_t* iuacc_reset;      /* [NIUA] */
    /* per-period analysis of a call (all NULL: off), after BubbleEnsemble.cu:174-216 */
    double* period_ref;              /* [UD][total_units] the state at the call's start */
    int32_t* period_number;          /* [total_units] first period (1-based) ending within period_tol of it, 0: none */
    double period_tol;
    double* max_accessory;           /* [total_units] running max of unit accessory max_accessory_index at period ends */
    int32_t max_accessory_index;
    int32_t n_sections;              /* Poincare sections stored per call */
    double* poincare;                /* [n_sections][total_units] state component 0 at the end of each period */
    int32_t band_width;              /* banded coupling storage (CBW > 0): the banded kernel variant's band */
    int32_t pad;
};

}  // namespace bes

#endif
