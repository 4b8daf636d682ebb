"""The golden cases: seeded ensembles run by the reference's own solver
(tests/golden/make_golden.py) and by the oracle (tests/test_oracle_golden.py)."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

from bubbleensemble_implicitextension_b200 import workloads as W

HERE = Path(__file__).resolve().parent


def _fixture_systems(name: str) -> list:
    """The systems a fixture was made for, as recorded in it (tests/golden/make_multiperiod.py
    chooses them: oracle-screened, then kept where the reference is not chaotic)."""
    f = HERE / f"{name}.npz"
    if not f.exists():
        return []
    return list(json.loads(str(np.load(f)["case"]))["systems"])

C1_SYSTEMS = [0, 2, 5, 18, 33, 47, 60, 85, 100, 128, 150, 175, 200, 222, 240, 255]

CASES = {
    "c1_n32": {"units": 32, "harness_ns": 256, "kind": "c1", "systems": C1_SYSTEMS},
    "c1_n32_do": {"units": 32, "harness_ns": 64, "kind": "c1", "systems": [33, 100, 175, 240]},
    "cloud_n64": {"units": 64, "harness_ns": 64, "kind": "cloud", "n_systems": 8, "seed": 64,
                  "pa_bar": 1.0, "f_khz": 120.0},
    "cloud_n128": {"units": 128, "harness_ns": 16, "kind": "cloud", "n_systems": 4, "seed": 128,
                   "pa_bar": 1.0, "f_khz": 150.0},
    # configuration 1's systems over 4 periods with the accessory reset before period 2
    "c1_n32_4p": {"units": 32, "harness_ns": 256, "kind": "c1", "systems": _fixture_systems("c1_n32_4p")},
}

RUNS = {
    "c1_n32": {"n_periods": 1, "reset_at": -1},
    "c1_n32_do": {"n_periods": 1, "reset_at": -1, "ndo": 16, "do_min_dt": 0.05, "do_save_frequency": 1},
    "cloud_n64": {"n_periods": 1, "reset_at": -1},
    "cloud_n128": {"n_periods": 1, "reset_at": -1},
    "c1_n32_4p": {"n_periods": 4, "reset_at": 1},
}

# fixtures written by their own script (screening and chaos check first)
MADE_ELSEWHERE = {"c1_n32_4p": "tests/golden/make_multiperiod.py"}

# cases with a fixture present (the multi-period one exists once make_multiperiod.py has run)
AVAILABLE = [n for n in CASES if (HERE / f"{n}.npz").exists() and (CASES[n].get("kind") != "c1" or CASES[n]["systems"])]
# the CPU oracle checks a bounded share of the long multi-period case (every 8th kept system);
# the GPU tests check every kept system
CPU_SUBSET = {"c1_n32_4p": slice(0, None, 8)}


def build(name: str, factored: bool = False, subset=None):
    """The case's ensemble with the reference-format coupling matrix (what the
    reference harness ran), or, factored, the same physics as a shared
    symmetric geometry with unit factors (the library's one-read kernels)."""
    spec, run = CASES[name], RUNS[name]
    if spec["kind"] == "c1":
        systems = spec["systems"] if subset is None else list(np.asarray(spec["systems"])[subset])
        ens = W.c1_ensemble(factored=factored).subset(systems)
    else:
        ens = W.c3_ensemble(n_systems=spec["n_systems"], n_units=spec["units"], seed=spec["seed"],
                            pa_bar=spec["pa_bar"], f_khz=spec["f_khz"], cube_um=400.0 * (spec["units"] / 32) ** (1 / 3),
                            n_periods=run["n_periods"], reset_at=run["reset_at"], factored=factored)
    ens.n_periods, ens.reset_at = run["n_periods"], run["reset_at"]
    return ens, run
