"""The oracle's single-reduction BiCG recurrence against the reference's own
solver (golden vectors), within the parity tolerances, and against the
reference recurrence on one right-hand side."""
import pytest

from tests import golden_compare
from tests.golden import cases


@pytest.mark.parametrize("name,factored", [(n, False) for n in cases.CASES] +
                         [(n, True) for n in ("c1_n32", "cloud_n64", "cloud_n128")])
def test_single_reduction_recurrence_matches_reference_golden(name, factored, oracle_lib):
    ens, run = cases.build(name, factored=factored)
    got = oracle_lib.run(ens, n_periods=run["n_periods"], reset_at=run["reset_at"], ndo=run.get("ndo", 0),
                         do_min_dt=run.get("do_min_dt", 0.0), do_save_frequency=run.get("do_save_frequency", 1),
                         bicg_variant=1)
    golden_compare.check(name, got)
