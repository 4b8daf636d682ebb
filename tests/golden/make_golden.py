"""Generate the golden fixtures from the reference's own CUDA solver.

Runs oracle/_ref (the reference's unmodified ProblemSolver, built by
oracle/build_ref.py for sm_100a) on seeded synthetic ensembles and stores its
outputs.  It needs a GPU and the prebuilt harness binaries; the inputs are
regenerated from the seeds recorded in each fixture, so a fixture holds only
the case description and the reference's outputs.

Cases (the reference is only well defined for N in {32, 64, 128} with
TPB = N, see its block reductions in
SourceCodes/CoupledSystems_PerBlock_ExplicitRungeKutta_Steppers.cuh:709-805):
  c1_n32      16 systems of the 1-D line ensemble, one period from rest,
              collapse events recorded;
  c1_n32_do   4 of those systems with 16 dense-output slots (radii at saved times);
  cloud_n64   8 systems sharing one random 3-D cloud of 64 bubbles, perturbed
              initial radii, one period;
  cloud_n128  4 systems sharing one random 3-D cloud of 128 bubbles, one period.

Usage (on the GPU machine):  python tests/golden/make_golden.py [outdir] [workdir]
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import build_ref, ref_io  # noqa: E402
from tests.golden import cases  # noqa: E402


def main(outdir: Path, work: Path) -> None:
    outdir.mkdir(parents=True, exist_ok=True)
    for name, spec in cases.CASES.items():
        if name in cases.MADE_ELSEWHERE:
            continue
        ens, run = cases.build(name)
        exe = build_ref.path(spec["units"], spec["harness_ns"], run.get("ndo", 0), True)
        out = ref_io.run(exe, ens, run["n_periods"], run["reset_at"], work, tag=name,
                         ndo=run.get("ndo", 0), do_min_dt=run.get("do_min_dt", 0.0),
                         do_save_frequency=run.get("do_save_frequency", 1))
        keep = {k: v for k, v in out.items() if isinstance(v, np.ndarray)}
        np.savez_compressed(outdir / f"{name}.npz", case=json.dumps({"name": name, **spec, **run}), **keep)
        print(f"{name}: {ens.n_systems} systems x {spec['units']} units, reference {out['elapsed_s']:.3f} s")


if __name__ == "__main__":
    # argv: [output directory for the .npz fixtures] [work directory for the harness's binary files]
    import tempfile
    main(Path(sys.argv[1]) if len(sys.argv) > 1 else Path(__file__).resolve().parent,
         Path(sys.argv[2]) if len(sys.argv) > 2 else Path(tempfile.gettempdir()) / "bes_golden_work")
