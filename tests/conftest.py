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


def rel_l1(a, b, floor_frac=1e-6):
    """relative L1 difference per conserved variable (axis 0).  A variable whose reference norm is
    below floor_frac of the largest variable's norm (an identically zero Bz) is measured against
    that floor instead of its own norm.  Residuals use floor_frac = 1e-2: a residual component can
    be pure cancellation (the density residual of Orszag-Tang, whose density is constant, is
    round-off of terms the size of the flux divergence), so it is measured on the residual's scale."""
    norms = np.array([np.abs(b[v]).sum() for v in range(b.shape[0])])
    floor = floor_frac * norms.max() if norms.max() > 0 else 1.0
    out = []
    for v in range(a.shape[0]):
        num = np.abs(a[v] - b[v]).sum()
        out.append(num / max(norms[v], floor))
    return np.array(out)
