import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN_DIR = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (run with -m gpu)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O

    O.lib()
    return O


@pytest.fixture(scope="session")
def native():
    """The product library, built for sm_100a (no CPU fallback)."""
    from shapeextraction_b200 import build

    build.build()
    from shapeextraction_b200 import _native

    _native.lib()
    return _native


def angle_deg_free(a, b):
    """Angle between unit vectors a and b in radians, ignoring sign."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    c = np.abs(np.sum(a * b, axis=1)) / (np.linalg.norm(a, axis=1) * np.linalg.norm(b, axis=1))
    return np.arccos(np.clip(c, -1.0, 1.0))
