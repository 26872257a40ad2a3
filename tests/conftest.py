import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# tensor-op (Ozaki) tests use small matrices: lower the size floor below which
# contractions stay on the plain FP64 path (read at library initialisation)
os.environ.setdefault("XKBLAS_OZAKI_MIN_DIM", "64")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")
    config.addinivalue_line("markers", "slow: large sizes, minutes of CPU")


@pytest.fixture(scope="session")
def xk():
    """The library under test, initialised on the GPU."""
    import xkblas_b200 as X
    X.init()
    yield X
    X.lib().xkblas_memory_invalidate_caches()


@pytest.fixture(scope="session")
def orc():
    import oracle as O
    O.lib()
    return O
