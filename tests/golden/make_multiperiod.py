"""Multi-period golden fixture from the reference's own CUDA solver.

Configuration 1's horizon runs many acoustic periods, with the accessory
reset between the transient and the recorded phase (CollapseStrength.cu:
123-147).  Past the first period some of its systems are chaotic, and some
drive the reference's step-size controller to the minimum step, where it
forces acceptance (ErrorControllers.cuh:525-529) and may need ~1e13 steps for
one period.  So the fixture is built in three stages:

1. Screen (CPU oracle): integrate all 256 systems of the 1-D line ensemble for
   N_PERIODS periods, accessories reset before period RESET_AT, with a budget
   of SCREEN_BUDGET attempted steps per period.  A system is a candidate when
   every period stays under the budget and its smallest attempted step stays
   above 1e3 x the minimum step size.  Only candidates are given to the
   reference, so the reference never meets a forced acceptance loop.
2. Chaos check (reference, on the GPU): run the candidates twice, with the
   equilibrium radii as drawn and with every radius raised by one ulp (unit
   parameters and coupling matrix recomputed).  A candidate is kept when the
   two runs agree to CHAOS_R on the final radii and dR/dtau (100x tighter
   than the parity bar of 1e-8), to CHAOS_S on the collapse strengths (10x
   tighter than the bar of 1e-6: a recorded minimum is the radius at an
   accepted step end, not a located extremum, so a shift of the step ends
   alone moves it by ~1e-8..1e-7 even where the dynamics do not diverge), with
   equal event counts; there, rounding-level differences between another FP64
   implementation and the reference stay below the bar.
3. The fixture keeps the reference's nominal outputs of the kept systems
   (tests/golden/c1_n32_4p.npz) together with the screening and chaos
   statistics of every system.

Usage (on the GPU machine):
    python tests/golden/make_multiperiod.py [outdir] [workdir]
"""
from __future__ import annotations

import dataclasses
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from bubbleensemble_implicitextension_b200 import workloads as W  # noqa: E402
from oracle import build_ref, ref_io  # noqa: E402
from oracle import oracle as O  # noqa: E402

N_PERIODS = 4
RESET_AT = 1
SCREEN_BUDGET = 20_000
CHAOS_R = 1e-10
CHAOS_S = 1e-7
NAME = "c1_n32_4p"


def screen(ens):
    """Per-period oracle run of every system; returns (candidate mask, stats)."""
    ns = ens.n_systems
    e = dataclasses.replace(ens, max_steps_per_period=SCREEN_BUDGET)
    state, uacc, iuacc = e.state.copy(), e.initial_uacc(), e.initial_iuacc()
    max_att = np.zeros(ns, np.int64)
    min_dt = np.full(ns, np.inf)
    status = np.zeros(ns, np.int32)
    for per in range(N_PERIODS):
        out = O.run(e, n_periods=1, reset_at=0 if per == RESET_AT else -1, state=state, uacc=uacc, iuacc=iuacc)
        state, uacc, iuacc = out["state"], out["uacc"], out["iuacc"]
        max_att = np.maximum(max_att, out["n_accepted"] + out["n_rejected"])
        min_dt = np.minimum(min_dt, out["min_dt"])
        status |= out["status"]
        print(f"screen: period {per} done, slowest system {int(max_att.max())} steps", flush=True)
    ok = (max_att < SCREEN_BUDGET) & (min_dt > 1e3 * ens.dtmin) & ((status & ~16) == 0)
    return ok, {"max_attempted_steps": max_att.tolist(), "min_dt": min_dt.tolist(), "status": status.tolist()}


def perturbed(ens):
    """The same ensemble with every equilibrium radius raised by one ulp."""
    info = ens.info
    radii = np.nextafter(info["radii_um"], np.inf)
    C = W.coupling_from_geometry(info["positions_um"], radii, info["cstr"])
    up = W.km_unit_parameters(info["pa_bar"][:, None], info["f_khz"][:, None], 0.0, 0.0, 0.0, radii[None, :])
    return dataclasses.replace(ens, upar=up.reshape(W.NUP, -1), coupling=C.T.reshape(-1).copy())


def chaos(a, b, units):
    """Per-system agreement of two runs: (max rel radius, max rel dR, max rel strength, equal counts)."""
    ns = len(units)
    R = np.abs(a["state"][0] - b["state"][0]) / np.abs(b["state"][0])
    dR = np.abs(a["state"][1] - b["state"][1]) / np.maximum(np.abs(b["state"][1]), 1.0)
    _, _, sa, ca = W.collapse_records(a["uacc"], a["iuacc"], units)
    _, _, sb, cb = W.collapse_records(b["uacc"], b["iuacc"], units)
    with np.errstate(divide="ignore", invalid="ignore"):
        S = np.where(sb > 0, np.abs(sa - sb) / np.abs(sb), np.where(sa > 0, np.inf, 0.0))
    n = int(units[0])
    Rs = R.reshape(ns, n).max(1)
    dRs = dR.reshape(ns, n).max(1)
    Ss = S.reshape(S.shape[0], ns, n).max(axis=(0, 2))
    same = (ca == cb).reshape(ns, n).all(1)
    return Rs, dRs, Ss, same


def subset_output(out, keep, n):
    """The reference's output arrays restricted to the kept systems (units contiguous, n per system)."""
    cols = np.concatenate([np.arange(s * n, (s + 1) * n) for s in keep])
    res = {"state": out["state"][:, cols], "uacc": out["uacc"][:, cols], "iuacc": out["iuacc"][:, cols],
           "actual_time": out["actual_time"][keep], "dense_index": out["dense_index"][keep],
           "period_s": out["period_s"]}
    return res


def main(outdir: Path, work: Path) -> None:
    ens = W.c1_ensemble(n_periods=N_PERIODS, reset_at=RESET_AT)
    ok, stats = screen(ens)
    cand = np.nonzero(ok)[0]
    print(f"screen: {len(cand)} of {ens.n_systems} systems are candidates", flush=True)
    exe = build_ref.path(32, 256, 0, True)
    sub = ens.subset(cand)
    sub.info = {k: (v[cand] if k in ("pa_bar", "f_khz") else v) for k, v in ens.info.items()}
    nominal = ref_io.run(exe, sub, N_PERIODS, RESET_AT, work, tag=NAME, timeout=3600)
    shifted = ref_io.run(exe, perturbed(sub), N_PERIODS, RESET_AT, work, tag=NAME + "_ulp", timeout=3600)
    Rs, dRs, Ss, same = chaos(nominal, shifted, sub.units)
    keep_mask = (Rs <= CHAOS_R) & (dRs <= CHAOS_R) & (Ss <= CHAOS_S) & same
    keep = np.nonzero(keep_mask)[0]
    systems = [int(cand[k]) for k in keep]
    print(f"chaos check: {len(systems)} of {len(cand)} candidates kept: {systems}", flush=True)
    g = subset_output(nominal, keep, 32)
    case = {"name": NAME, "units": 32, "harness_ns": 256, "kind": "c1", "systems": systems,
            "n_periods": N_PERIODS, "reset_at": RESET_AT,
            "screen": {"budget": SCREEN_BUDGET, "min_dt_factor": 1e3, "candidates": cand.tolist(), **stats},
            "chaos": {"radius": Rs.tolist(), "dR": dRs.tolist(), "strength": [float(x) for x in Ss],
                      "equal_counts": same.tolist(), "tol_radius": CHAOS_R, "tol_strength": CHAOS_S},
            "reference_seconds": float(nominal["elapsed_s"])}
    outdir.mkdir(parents=True, exist_ok=True)
    np.savez_compressed(outdir / f"{NAME}.npz", case=json.dumps(case), **g)
    print(f"{NAME}: {len(systems)} systems, reference {nominal['elapsed_s']:.1f} s", flush=True)


if __name__ == "__main__":
    import tempfile
    main(Path(sys.argv[1]) if len(sys.argv) > 1 else Path(__file__).resolve().parent,
         Path(sys.argv[2]) if len(sys.argv) > 2 else Path(tempfile.gettempdir()) / "bes_golden_work")
