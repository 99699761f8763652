"""Shared test setup: the `gpu` marker, import paths, and helpers that build the compared scenes."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 CUDA device")


def has_gpu():
    try:
        from photon_b200 import native
        return native.device_info() is not None
    except ImportError:
        return False


@pytest.fixture(scope="session")
def gpu_available():
    return has_gpu()


@pytest.fixture
def require_gpu():
    if not has_gpu():
        pytest.skip("no CUDA device")


def pixel_agreement(a, b):
    """Photon's GPU-vs-CPU comparison (tests/test_gpu.cpp:58-68): the fraction of pixels whose
    largest channel difference is within 1e-3 * max(1, max channel of the reference), and the two
    mean luminances."""
    d = np.abs(a - b).max(axis=-1)
    tol = 1e-3 * np.maximum(1.0, a.max(axis=-1))
    frac = float((d <= tol).mean())
    lum = np.array([0.2126, 0.7152, 0.0722], np.float64)
    return frac, float((a.astype(np.float64) @ lum).mean()), float((b.astype(np.float64) @ lum).mean())
