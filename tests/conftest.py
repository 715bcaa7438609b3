"""Shared fixtures.  GPU tests are marked ``gpu``; everything else runs on CPU.

The oracle (``oracle/``) is the checker only: tests compare the CUDA library,
called through its C ABI, against it.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle as O
    return O.Oracle()


@pytest.fixture(scope="session")
def clarity_gpu():
    """The registered CUDA library (GPU tests only)."""
    from clarity_b200 import api
    api.load()
    api.register()
    yield api
    api.unregister()


def load_golden(name):
    path = os.path.join(GOLDEN, name + ".npz")
    return dict(np.load(path))


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0))
