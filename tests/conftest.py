"""Shared fixtures.  GPU tests are marked ``gpu``; everything else runs on CPU.

The oracle (``oracle/``) is the checker only: tests compare the CUDA library,
called through its C ABI, against it.
"""
import hashlib
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")
# Reference outputs at the full workload sizes (tens of MB each): computed by
# the reference's CPU build or the FP64 oracle on first use and kept here,
# outside version control, keyed by the inputs' digest.
LARGE = os.path.join(GOLDEN, "_large")


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


def cached(name, inputs, fn):
    """fn()'s array, computed once per (name, inputs) and kept under
    tests/golden/_large (the CPU reference at full size takes seconds to
    minutes; the key includes a digest of every input array)."""
    h = hashlib.sha1()
    for a in inputs:
        h.update(np.ascontiguousarray(a).tobytes())
    path = os.path.join(LARGE, f"{name}-{h.hexdigest()[:16]}.npy")
    if os.path.exists(path):
        return np.load(path)
    out = fn()
    try:
        os.makedirs(LARGE, exist_ok=True)
        np.save(path + ".tmp.npy", out)
        os.replace(path + ".tmp.npy", path)
    except OSError:
        pass
    return out


_REPORT = {}


def report_error(name, **values):
    """Records a result's errors; written as JSON at the end of the session to
    the file $CLARITY_PARITY_REPORT names (when set)."""
    _REPORT[name] = {k: float(v) for k, v in values.items()}


def pytest_sessionfinish(session, exitstatus):
    path = os.environ.get("CLARITY_PARITY_REPORT")
    if path and _REPORT:
        with open(path, "w") as f:
            json.dump(_REPORT, f, indent=1, sort_keys=True)


@pytest.fixture(scope="session")
def ref_cpu():
    """The reference's own CPU build with a double flux sum (oracle/_ref),
    all host threads; None where it was not built (the oracle's FP32
    restatement, pinned bit-identical to it, stands in)."""
    import oracle as O
    if not O.ReferenceCPU.available("ref_fp64sum"):
        return None
    r = O.ReferenceCPU("ref_fp64sum")
    r.set_threads(os.cpu_count() or 1)
    return r
