import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the CUDA kernels through the C ABI)")


@pytest.fixture(scope="session")
def mq():
    """The package, initialised on cuda:0 (GPU tests only)."""
    import mossquantum_b200 as m
    m.init(0)
    return m


@pytest.fixture(scope="session")
def O():
    from oracle import oracle
    oracle.set_threads(min(8, os.cpu_count() or 1))
    return oracle
