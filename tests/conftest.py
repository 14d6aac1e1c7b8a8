import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session")
def oracle():
    from oracle import binding
    binding.lib()
    return binding


@pytest.fixture(scope="session")
def sb():
    """The product package with its CUDA library loaded (built if missing)."""
    from sciwasm.sparse_b200 import build as _build
    _build.build()
    import sciwasm.sparse_b200 as pkg
    pkg.load_library()
    return pkg


@pytest.fixture(scope="session")
def gpu(sb):
    """Session fixture for GPU tests: fails (does not skip) without a device."""
    import ctypes
    from sciwasm.sparse_b200 import _lib
    n = ctypes.c_int(0)
    _lib.call("sb_device_count", ctypes.byref(n))
    assert n.value > 0, "GPU test collected but no CUDA device is visible"
    return sb


def rel_err(y, truth):
    y = np.asarray(y, dtype=np.float64)
    t = np.asarray(truth, dtype=np.float64)
    den = np.max(np.abs(t)) if t.size else 0.0
    if den == 0.0:
        return float(np.max(np.abs(y - t))) if t.size else 0.0
    return float(np.max(np.abs(y - t)) / den)


TOL = {np.dtype(np.float32): 1e-5, np.dtype(np.float64): 1e-12}
