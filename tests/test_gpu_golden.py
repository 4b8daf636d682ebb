"""The CUDA kernel against the reference's own solver (golden vectors)."""
import pytest

from tests import golden_compare
from tests.golden import cases
from tests.helpers import run_gpu

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", cases.AVAILABLE)
def test_kernel_matches_reference_golden(name, gpu):
    ens, run = cases.build(name)
    got = run_gpu(ens, n_periods=run["n_periods"], reset_at=run["reset_at"], ndo=run.get("ndo", 0),
                  do_min_dt=run.get("do_min_dt", 0.0), do_save_frequency=run.get("do_save_frequency", 1))
    golden_compare.check(name, got)


@pytest.mark.parametrize("name", [n for n in ("c1_n32", "cloud_n64", "cloud_n128", "c1_n32_4p")
                                  if n in cases.AVAILABLE])
def test_symmetric_geometry_kernels_match_reference_golden(name, gpu):
    """The same systems as a shared symmetric geometry with unit factors (row of
    G in registers for N = 32, one shared-memory read for both products above)
    against the reference's own solver run on the reference-format matrix."""
    ens, run = cases.build(name, factored=True)
    got = run_gpu(ens, n_periods=run["n_periods"], reset_at=run["reset_at"])
    golden_compare.check(name, got)
