"""The oracle's single-reduction BiCG recurrence against the reference's own
solver (golden vectors), within the parity tolerances, and against the
reference recurrence on one right-hand side."""
import pytest

from tests import golden_compare
from tests.golden import cases


@pytest.mark.parametrize("name,factored", [(n, False) for n in cases.AVAILABLE] +
                         [(n, True) for n in ("c1_n32", "cloud_n64", "cloud_n128")])
def test_single_reduction_recurrence_matches_reference_golden(name, factored, oracle_lib):
    sub = None if factored else cases.CPU_SUBSET.get(name)
    ens, run = cases.build(name, factored=factored, subset=sub)
    got = oracle_lib.run(ens, n_periods=run["n_periods"], reset_at=run["reset_at"], ndo=run.get("ndo", 0),
                         do_min_dt=run.get("do_min_dt", 0.0), do_save_frequency=run.get("do_save_frequency", 1),
                         bicg_variant=1)
    golden_compare.check(name, got, subset=sub, multi_period_share=5e-3)
