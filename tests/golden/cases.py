"""The golden cases: seeded ensembles run by the reference's own solver
(tests/golden/make_golden.py) and by the oracle (tests/test_oracle_golden.py)."""
from __future__ import annotations

import numpy as np

from bubbleensemble_implicitextension_b200 import workloads as W

C1_SYSTEMS = [0, 2, 5, 18, 33, 47, 60, 85, 100, 128, 150, 175, 200, 222, 240, 255]

CASES = {
    "c1_n32": {"units": 32, "harness_ns": 256, "kind": "c1", "systems": C1_SYSTEMS},
    "c1_n32_do": {"units": 32, "harness_ns": 64, "kind": "c1", "systems": [33, 100, 175, 240]},
    "cloud_n64": {"units": 64, "harness_ns": 64, "kind": "cloud", "n_systems": 8, "seed": 64,
                  "pa_bar": 1.0, "f_khz": 120.0},
    "cloud_n128": {"units": 128, "harness_ns": 16, "kind": "cloud", "n_systems": 4, "seed": 128,
                   "pa_bar": 1.0, "f_khz": 150.0},
}

RUNS = {
    "c1_n32": {"n_periods": 1, "reset_at": -1},
    "c1_n32_do": {"n_periods": 1, "reset_at": -1, "ndo": 16, "do_min_dt": 0.05, "do_save_frequency": 1},
    "cloud_n64": {"n_periods": 1, "reset_at": -1},
    "cloud_n128": {"n_periods": 1, "reset_at": -1},
}


def build(name: str, factored: bool = False):
    """The case's ensemble with the reference-format coupling matrix (what the
    reference harness ran), or, factored, the same physics as a shared
    symmetric geometry with unit factors (the library's one-read kernels)."""
    spec, run = CASES[name], RUNS[name]
    if spec["kind"] == "c1":
        ens = W.c1_ensemble(factored=factored).subset(spec["systems"])
    else:
        ens = W.c3_ensemble(n_systems=spec["n_systems"], n_units=spec["units"], seed=spec["seed"],
                            pa_bar=spec["pa_bar"], f_khz=spec["f_khz"], cube_um=400.0 * (spec["units"] / 32) ** (1 / 3),
                            n_periods=run["n_periods"], reset_at=run["reset_at"], factored=factored)
    ens.n_periods, ens.reset_at = run["n_periods"], run["reset_at"]
    return ens, run
