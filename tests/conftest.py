import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA library")
    config.addinivalue_line("markers", "slow: long-running check")


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import oracle as O
    O.build()
    return O.load()


@pytest.fixture(scope="session")
def built_libs():
    """The CUDA libraries, built in-tree (nvcc cross-compiles without a GPU)."""
    from fluidphysics_b200 import build as B
    return B.build()
