import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def lib():
    """The CUDA library (built in-tree if missing)."""
    import elfmmlib3d_b200 as E
    if not os.path.exists(E.library_path()):
        from elfmmlib3d_b200 import build
        build.build()
    E.load()
    return E


@pytest.fixture(scope="session")
def gpu(lib):
    if lib.device_count() < 1:
        pytest.fail("GPU test run without a visible CUDA device")
    return lib


def golden(name):
    return dict(np.load(os.path.join(GOLDEN, name)))


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))
