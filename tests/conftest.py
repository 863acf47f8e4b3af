import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs on the B200 box)")


def rel_err(got, ref, floor=1e-12):
    """Per-point relative error with a floor relative to the largest |ref|."""
    got = np.asarray(got)
    ref = np.asarray(ref)
    scale = np.max(np.abs(ref)) if ref.size else 1.0
    return np.abs(got - ref) / np.maximum(np.abs(ref), floor * scale)


@pytest.fixture(scope="session")
def oracle():
    from oracle import build as ob
    ob.build()
    from oracle import oracle as O
    return O
