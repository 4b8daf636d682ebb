"""Fault-injection cases for the per-system status word.

Each case makes a failure on the host side -- a NaN in one unit's
parameters, a tiny step budget, a minimum step above the initial step, a
minimum step that no event cut can reach -- and states which status bits the
reference's controller and event logic then produce
(ErrorControllers.cuh:512-529, EventHandling.cuh:257-266).  The solver never
traps and every case ends in a bounded number of steps: a non-finite step
shrinks dt to the minimum and terminates the system, the step budget ends the
period, forced acceptance at the minimum step advances time."""
import dataclasses

import numpy as np

from bubbleensemble_implicitextension_b200 import workloads as W

NONFINITE, MIN_STEP, STEP_BUDGET, EVENT_MISSED, BICG_CAP = 1, 2, 4, 8, 16


def base():
    ens = W.c1_ensemble().subset([10, 100, 250])
    ens.max_steps_per_period = 50_000
    return ens


def nan_parameter():
    """System 1, unit 7: unit parameter 5 (the drive amplitude term) is NaN."""
    e = base()
    e = dataclasses.replace(e, upar=e.upar.copy())
    e.upar[5, 32 + 7] = np.nan
    return e


def step_budget():
    return dataclasses.replace(base(), max_steps_per_period=50)


def min_step_above_initial():
    return dataclasses.replace(base(), dt0=1e-3, dtmin=2e-3)


def unreachable_event_cut():
    return dataclasses.replace(base(), dtmin=1e-5)


# name -> (ensemble builder, {system: bits that must be set}, {system: bits that must be clear})
CASES = {
    "nan_parameter": (nan_parameter, {1: NONFINITE}, {0: NONFINITE, 2: NONFINITE}),
    "step_budget": (step_budget, {0: STEP_BUDGET, 1: STEP_BUDGET, 2: STEP_BUDGET}, {}),
    "min_step_above_initial": (min_step_above_initial, {0: MIN_STEP, 1: MIN_STEP, 2: MIN_STEP}, {}),
    "unreachable_event_cut": (unreachable_event_cut, {1: EVENT_MISSED, 2: EVENT_MISSED}, {1: NONFINITE, 2: NONFINITE}),
}


def check_bits(status, must, must_not):
    for s, bits in must.items():
        assert status[s] & bits == bits, f"system {s}: status {status[s]} lacks bits {bits}"
    for s, bits in must_not.items():
        assert status[s] & bits == 0, f"system {s}: status {status[s]} has bits {bits}"
