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
    golden_compare.check(name, got, subset=sub)


@pytest.mark.parametrize("factored,systems", [(True, [1, 7]), (False, [13])])
def test_safeguard_replaces_broken_down_solves(factored, systems, oracle_lib):
    """Systems of configuration 1 on which the unguarded single-reduction
    recurrence broke down (non-finite state, the system terminated): with the
    true-residual check the failing solves are redone with the reference's
    recurrence, nothing goes non-finite, and the radii agree with the
    reference recurrence's run to the parity bar."""
    import numpy as np

    from bubbleensemble_implicitextension_b200 import workloads as W
    ens = W.c1_ensemble(n_periods=1, reset_at=-1, factored=factored).subset(systems)
    L = oracle_lib.lib()
    L.bes_oracle_rec1_fallbacks(1)
    a = oracle_lib.run(ens, n_periods=1, reset_at=-1, bicg_variant=1)
    assert L.bes_oracle_rec1_fallbacks(1) > 0
    b = oracle_lib.run(ens, n_periods=1, reset_at=-1, bicg_variant=0)
    assert (a["status"] & 1 == 0).all()
    np.testing.assert_array_equal(a["iuacc"], b["iuacc"])
    assert (np.abs(a["state"][0] - b["state"][0]) / b["state"][0]).max() < 1e-8
