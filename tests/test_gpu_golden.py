"""The CUDA kernel against the reference's own solver (golden vectors)."""
import pytest

from tests import golden_compare
from tests.golden import cases
from tests.helpers import run_gpu

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", list(cases.CASES))
def test_kernel_matches_reference_golden(name, gpu):
    ens, run = cases.build(name)
    got = run_gpu(ens, n_periods=run["n_periods"], reset_at=run["reset_at"], ndo=run.get("ndo", 0),
                  do_min_dt=run.get("do_min_dt", 0.0), do_save_frequency=run.get("do_save_frequency", 1))
    golden_compare.check(name, got)
