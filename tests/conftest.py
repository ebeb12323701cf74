import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import __graft_entry__  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def pkg():
    __graft_entry__._build_module().build()
    return __graft_entry__.load_package()


@pytest.fixture(scope="session")
def ora():
    from oracle import oracle
    return oracle


def rel_l1(a, b):
    """relative L1 difference per conserved variable (axis 0); absolute where the reference is 0"""
    out = []
    for v in range(a.shape[0]):
        den = np.abs(b[v]).sum()
        num = np.abs(a[v] - b[v]).sum()
        out.append(num / den if den > 0 else num)
    return np.array(out)
