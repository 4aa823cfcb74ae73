"""Shared pytest configuration.

`-m gpu` tests need a B200 and the in-tree CUDA library; `-m "not gpu"` tests run
on CPU only (oracle vs golden vectors, host logic, C-ABI symbol table).
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built library")
    config.addinivalue_line("markers", "slow: longer statistical runs")


def load_golden(name):
    path = os.path.join(GOLDEN, name)
    with np.load(path, allow_pickle=False) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="session")
def golden():
    return load_golden


@pytest.fixture(scope="session")
def md():
    """The product library; fails loudly (never skips) when it is not built."""
    import moleculardynamics_b200 as mdb
    mdb.require_gpu()
    return mdb
