import os
import sys

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
PKG = os.path.join(ROOT, "phyflow2.0_b200")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests through the C ABI")


@pytest.fixture(scope="session")
def golden():
    def load(name):
        return dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    return load


def normwise_err(vx, vy, rx, ry):
    """max_i |v_i - v_ref_i| / max_i |v_ref_i| (vector norm per point)."""
    d = np.sqrt((np.asarray(vx) - rx) ** 2 + (np.asarray(vy) - ry) ** 2)
    return float(d.max() / np.sqrt(rx * rx + ry * ry).max())
