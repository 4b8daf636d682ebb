"""Fault injection on the GPU: host-made failures (NaN parameters, a tiny step
budget, a minimum step above the initial step, an unreachable event cut) end
in bounded time with the status bits of the reference's controller and event
logic, bit-identical to the oracle -- states, counters and status words."""
import pytest

from tests import status_cases as SC
from tests.helpers import assert_bitwise, run_gpu

pytestmark = pytest.mark.gpu

KEYS = ["state", "uacc", "iuacc", "n_accepted", "n_rejected", "n_bicg_iter", "n_rhs", "status"]


@pytest.mark.parametrize("rec", [0, 1])
@pytest.mark.parametrize("name", list(SC.CASES))
def test_status_bits_match_oracle(name, rec, gpu, oracle_lib):
    build, must, must_not = SC.CASES[name]
    ens = build()
    got = run_gpu(ens, n_periods=1, reset_at=-1, bicg_recurrence=rec)
    want = oracle_lib.run(ens, n_periods=1, reset_at=-1, bicg_variant=rec)
    assert_bitwise(got, want, KEYS)
    SC.check_bits(got["status"], must, must_not)
