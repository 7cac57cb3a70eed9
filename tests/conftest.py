import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "cuda-orb_b200")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def canon_order(points):
    """Order that sorts keypoints by (y, x); NMS leaves at most one per pixel."""
    return np.lexsort((points["x"], points["y"]))


def load_golden(name):
    path = os.path.join(GOLDEN, name)
    if not os.path.exists(path):
        pytest.skip(f"missing fixture {name}")
    return np.load(path)


@pytest.fixture(scope="session")
def golden():
    return load_golden
