"""The oracle's status bits under host-injected failures (the CPU side of the
fault-injection tests; tests/test_gpu_status.py runs the same cases on the GPU)."""
import numpy as np
import pytest

from tests import status_cases as SC


@pytest.mark.parametrize("name", list(SC.CASES))
def test_oracle_status_bits(name, oracle_lib):
    build, must, must_not = SC.CASES[name]
    ens = build()
    out = oracle_lib.run(ens, n_periods=1, reset_at=-1)
    SC.check_bits(out["status"], must, must_not)
    attempted = out["n_accepted"] + out["n_rejected"]
    assert (attempted <= ens.max_steps_per_period).all()


def test_nan_parameter_leaves_the_other_systems_untouched(oracle_lib):
    clean = oracle_lib.run(SC.base(), n_periods=1, reset_at=-1)
    bad = oracle_lib.run(SC.nan_parameter(), n_periods=1, reset_at=-1)
    for s in (0, 2):
        cols = slice(32 * s, 32 * (s + 1))
        np.testing.assert_array_equal(bad["state"][:, cols], clean["state"][:, cols])
        assert bad["status"][s] == clean["status"][s]
