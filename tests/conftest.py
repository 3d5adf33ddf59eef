import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libsurfatt_gpu.so")
    config.addinivalue_line("markers", "slow: long-running parity case")


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def gpu():
    """The product library on cuda:0; fails loudly if it cannot load."""
    from surfattpp_b200 import _capi
    _capi.lib()
    return _capi.default_context()


def lin(n, a, b):
    return np.linspace(a, b, n)
