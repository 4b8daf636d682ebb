"""Drop-in: the driver that runs the reference's ProblemSolver
(oracle/ref_harness.cu) compiled unchanged against include/dropin/ (the C++
ProblemSolver shim over libbes.so).  Its results must be bit-identical to
the library driven from Python and within tolerance of the reference."""
import numpy as np
import pytest

from oracle import build_ref, ref_io
from tests import golden_compare
from tests.golden import cases
from tests.helpers import assert_bitwise, run_gpu

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["c1_n32", "c1_n32_do"])
def test_reference_driver_runs_on_the_library(name, gpu, tmp_path):
    ens, run = cases.build(name)
    ndo = run.get("ndo", 0)
    exe = build_ref.dropin_path(32, 64 if ndo else 256, ndo)
    if not exe.exists():
        build_ref.build_dropin()
    out = ref_io.run(exe, ens, run["n_periods"], run["reset_at"], tmp_path, tag=name, ndo=ndo,
                     do_min_dt=run.get("do_min_dt", 0.0), do_save_frequency=run.get("do_save_frequency", 1))
    golden_compare.check(name, out)
    direct = run_gpu(ens, n_periods=run["n_periods"], reset_at=run["reset_at"], ndo=ndo,
                     do_min_dt=run.get("do_min_dt", 0.0), do_save_frequency=run.get("do_save_frequency", 1))
    keys = ["state", "uacc", "iuacc"] + (["dense_index", "dense_time", "dense_state"] if ndo else [])
    assert_bitwise(out, direct, keys)
