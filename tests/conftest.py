import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the sm_100a library")
    config.addinivalue_line("markers", "slow: long-running CPU test")


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def bes_lib():
    """The product library; on a GPU machine a missing build is an error, never a fallback."""
    from bubbleensemble_implicitextension_b200 import _build
    _build.build()
    from bubbleensemble_implicitextension_b200 import solver
    return solver.load_library()


@pytest.fixture(scope="session")
def gpu(bes_lib):
    from bubbleensemble_implicitextension_b200 import solver
    n = solver.device_count()
    if n < 1:
        pytest.fail("a GPU test ran without a visible CUDA device")
    return 0
