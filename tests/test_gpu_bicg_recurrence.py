"""The single-reduction BiCG recurrence (BiCGRecurrence = 1) on the GPU.

Kernel against the oracle's restatement of the same recurrence, bit for bit,
on every kernel layout (register-resident operators for N <= 32, the
operator in shared memory, staged shared matrices with and without
symmetry, one and several warps per system), and kernel against the
reference's own solver (golden vectors) within the parity tolerances
(radii 1e-8, collapse strength 1e-6, equal event counts; over several
periods the rule of tests/golden_compare.py): the recurrence produces the
reference's iterates in exact arithmetic and rounds differently.  The
systems on which the unguarded recurrence broke down run bit-identical to
the oracle and stay finite (the true-residual safeguard)."""
import numpy as np
import pytest

from bubbleensemble_implicitextension_b200 import workloads as W
from tests import golden_compare
from tests.golden import cases
from tests.helpers import assert_bitwise, ragged_ensemble, run_gpu

pytestmark = pytest.mark.gpu

KEYS = ["state", "uacc", "iuacc", "n_accepted", "n_rejected", "n_bicg_iter", "n_rhs", "status"]
REC = 1


def bounded(ens, budget=50_000):
    ens.max_steps_per_period = budget
    return ens


@pytest.mark.parametrize("factored", [False, True])
def test_c1_subset_matches_oracle(gpu, oracle_lib, factored):
    """N = 32: register-resident W (reference-format matrix) or row of G (geometry with factors)."""
    ens = bounded(W.c1_ensemble(factored=factored).subset([0, 9, 64, 131, 200, 255]))
    got = run_gpu(ens, n_periods=2, reset_at=1, bicg_recurrence=REC)
    want = oracle_lib.run(ens, n_periods=2, reset_at=1, bicg_variant=REC)
    assert_bitwise(got, want, KEYS)


@pytest.mark.parametrize("wps", [0, 1])
def test_ragged_matches_oracle(gpu, oracle_lib, wps):
    """Operator W in shared memory, N from 4 to 128, on groups of warps (0) or single warps (1)."""
    ens = bounded(ragged_ensemble([4, 17, 32, 33, 48, 64, 100, 128], seed=21))
    got = run_gpu(ens, n_periods=1, reset_at=-1, bicg_recurrence=REC, warps_per_system=wps)
    want = oracle_lib.run(ens, n_periods=1, reset_at=-1, bicg_variant=REC)
    assert_bitwise(got, want, KEYS)


@pytest.mark.parametrize("factored,wps", [(False, 0), (True, 0), (True, 1)])
def test_shared_matrix_n128_matches_oracle(gpu, oracle_lib, factored, wps):
    """One staged matrix per CTA: unsymmetric (column tree) and symmetric (one read for both products)."""
    ens = bounded(W.c3_ensemble(n_systems=6, n_units=128, n_periods=1, reset_at=-1, factored=factored))
    got = run_gpu(ens, n_periods=1, reset_at=-1, bicg_recurrence=REC, warps_per_system=wps)
    want = oracle_lib.run(ens, n_periods=1, reset_at=-1, bicg_variant=REC)
    assert_bitwise(got, want, KEYS)


def test_dense_output_and_cap_match_oracle(gpu, oracle_lib):
    """Dense output, and a BiCG cap of 3 iterations (the capped exit path and its status bit)."""
    ens = bounded(W.c1_ensemble().subset([40, 41]))
    got = run_gpu(ens, n_periods=1, reset_at=-1, ndo=12, do_min_dt=0.05, bicg_recurrence=REC, bicg_max_iter=3)
    want = oracle_lib.run(ens, n_periods=1, reset_at=-1, ndo=12, do_min_dt=0.05, bicg_variant=REC, bicg_max_iter=3)
    assert_bitwise(got, want, KEYS + ["dense_index", "dense_time", "dense_state"])
    assert (got["status"] & 16).any(), "the cap of 3 iterations was never reached"


@pytest.mark.parametrize("name", cases.AVAILABLE)
def test_matches_reference_golden(gpu, name):
    ens, run = cases.build(name)
    got = run_gpu(ens, n_periods=run["n_periods"], reset_at=run["reset_at"], ndo=run.get("ndo", 0),
                  do_min_dt=run.get("do_min_dt", 0.0), do_save_frequency=run.get("do_save_frequency", 1),
                  bicg_recurrence=REC)
    golden_compare.check(name, got)


@pytest.mark.parametrize("name", [n for n in ("c1_n32", "cloud_n64", "cloud_n128", "c1_n32_4p")
                                  if n in cases.AVAILABLE])
def test_factored_matches_reference_golden(gpu, name):
    ens, run = cases.build(name, factored=True)
    got = run_gpu(ens, n_periods=run["n_periods"], reset_at=run["reset_at"], bicg_recurrence=REC)
    golden_compare.check(name, got)


@pytest.mark.parametrize("factored,systems", [(True, [1, 7]), (False, [13])])
def test_safeguard_matches_oracle_where_the_recurrence_broke_down(gpu, oracle_lib, factored, systems):
    ens = bounded(W.c1_ensemble(factored=factored).subset(systems))
    got = run_gpu(ens, n_periods=1, reset_at=-1, bicg_recurrence=REC)
    want = oracle_lib.run(ens, n_periods=1, reset_at=-1, bicg_variant=REC)
    assert_bitwise(got, want, KEYS)
    assert (got["status"] & 1 == 0).all()
