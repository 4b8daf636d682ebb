"""The banded operator (banded coupling storage, CBW > 0: only the wrapping
band of 2 CBW + 1 diagonals couples, ExplicitRungeKutta_Steppers.cuh:586-641)
on the GPU against the oracle's banded association, bit for bit: rings of
bubbles coupled to their CBW neighbours on either side, one warp (N <= 32),
two or four warps per system, both BiCG recurrences, and a band as wide as
the system (every column once, in band order)."""
import numpy as np
import pytest

from bubbleensemble_implicitextension_b200 import workloads as W
from tests.helpers import assert_bitwise, run_gpu

pytestmark = pytest.mark.gpu

KEYS = ["state", "uacc", "iuacc", "n_accepted", "n_rejected", "n_bicg_iter", "n_rhs", "status"]


@pytest.mark.parametrize("rec", [0, 1])
@pytest.mark.parametrize("n,bw", [(20, 3), (64, 2), (128, 1), (128, 7), (8, 5)])
def test_banded_ring_matches_oracle(n, bw, rec, gpu, oracle_lib):
    ens = W.ring_ensemble(n_systems=5, n_units=n, band_width=bw)
    ens.max_steps_per_period = 50_000
    got = run_gpu(ens, n_periods=1, reset_at=-1, bicg_recurrence=rec)
    want = oracle_lib.run(ens, n_periods=1, reset_at=-1, bicg_variant=rec)
    assert_bitwise(got, want, KEYS)


def test_banded_ragged_sizes_one_launch_per_class(gpu, oracle_lib):
    """Systems of 12, 40 and 100 units in one solve: the banded operator in every size class."""
    parts = [W.ring_ensemble(n_systems=2, n_units=n, band_width=2, seed=s) for s, n in ((1, 12), (2, 40), (3, 100))]
    ens = W.Ensemble(units=np.concatenate([p.units for p in parts]), upar=np.concatenate([p.upar for p in parts], 1),
                     state=np.concatenate([p.state for p in parts], 1),
                     coupling=np.concatenate([p.coupling for p in parts]),
                     matrix_of_system=np.arange(6, dtype=np.int32), rtol=np.full((2, 6), 1e-10),
                     atol=np.full((2, 6), 1e-10), n_periods=1, reset_at=-1, band_width=2, max_steps_per_period=50_000)
    got = run_gpu(ens, n_periods=1, reset_at=-1)
    want = oracle_lib.run(ens, n_periods=1, reset_at=-1)
    assert_bitwise(got, want, KEYS)
