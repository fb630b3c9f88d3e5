import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests of the CUDA path")


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle as orc
    orc.build()
    return orc


@pytest.fixture(scope="session")
def gpu_lib():
    """The CUDA library, built in-tree; fails loudly if it cannot load."""
    from dense_hodlr_b200 import _lib
    from dense_hodlr_b200 import build as b
    b.build()
    return _lib.lib()


def c1_points(n=4096, seed=1):
    rng = np.random.default_rng(seed)
    return np.sort(rng.uniform(-1.0, 1.0, n))[None, :], rng
