/* bes_status.h -- per-system status bits written by the solver kernel. */
#ifndef BES_STATUS_H
#define BES_STATUS_H

/* The reference only printf()s these conditions from the device
 * (SourceCodes/CoupledSystems_PerBlock_ExplicitRungeKutta_ErrorControllers.cuh:519,527,
 * SourceCodes/CoupledSystems_PerBlock_EventHandling.cuh:260); here they are
 * recorded per system and returned to the host. */
#define BES_STATUS_NONFINITE 1      /* terminated: state not finite at the minimum step */
#define BES_STATUS_MIN_STEP 2       /* a step was forced through at the minimum step size */
#define BES_STATUS_STEP_BUDGET 4    /* the per-period step budget ran out (the period was cut short) */
#define BES_STATUS_EVENT_MISSED 8   /* an event cut would have gone below the minimum step; not located */
#define BES_STATUS_BICG_CAP 16      /* a BiCG solve used all its iterations without meeting an exit test */

#endif
