"""The oracle against golden vectors from the reference's own CUDA solver.

tests/golden/*.npz were written by tests/golden/make_golden.py, which ran
the reference's unmodified ProblemSolver (built for sm_100a from its own
headers by oracle/build_ref.py) on a B200.  This pins the oracle: the
oracle must reproduce the reference within the parity tolerances."""
import pytest

from tests import golden_compare
from tests.golden import cases


@pytest.mark.parametrize("name", cases.AVAILABLE)
def test_oracle_matches_reference_golden(name, oracle_lib):
    sub = cases.CPU_SUBSET.get(name)
    ens, run = cases.build(name, subset=sub)
    got = oracle_lib.run(ens, n_periods=run["n_periods"], reset_at=run["reset_at"], ndo=run.get("ndo", 0),
                         do_min_dt=run.get("do_min_dt", 0.0), do_save_frequency=run.get("do_save_frequency", 1))
    golden_compare.check(name, got, subset=sub)


def test_golden_fixtures_present():
    for name in cases.AVAILABLE:
        g, case = golden_compare.load(name)
        assert case["name"] == name and "state" in g and "uacc" in g
