import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built CUDA library")


GOLDEN = os.path.join(ROOT, "tests", "golden")


@pytest.fixture(scope="session")
def golden_dir():
    return GOLDEN

PKG = os.path.join(ROOT, "exafmm-t_b200")
if PKG not in sys.path:
    sys.path.insert(0, PKG)

# load the library (and the CUDA libraries it was built with) before any test module imports torch,
# as bench.py does; a missing build is reported by the tests themselves
try:
    import exafmm  # noqa: F401
except ImportError:
    pass
