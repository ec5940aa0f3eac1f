"""Test configuration.

Markers:
    gpu -- needs a CUDA device (B200); these are the parity tests of the CUDA path proper and call
           it through the C ABI (libpvb200.so). Everything unmarked runs on a CPU-only machine.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device; parity tests of the CUDA path")


@pytest.fixture(scope="session")
def port():
    """The C restatement of the reference (oracle/pv_oracle.c)."""
    from oracle import pyoracle
    if not os.path.exists(pyoracle.PORT_LIB):
        pyoracle.build(reference=False)
    return pyoracle.Oracle("port")


@pytest.fixture(scope="session")
def reference():
    """The unmodified reference compiled into oracle/_ref/ (skipped when it was not built)."""
    from oracle import pyoracle
    if not os.path.exists(pyoracle.REF_LIB):
        pytest.skip("oracle/_ref/libpvref.so was not built (reference sources absent)")
    return pyoracle.Oracle("reference")


def golden(name: str):
    return np.load(os.path.join(GOLDEN, name))


def normalized_error(u, v, ur, vr) -> np.ndarray:
    """Per-vortex velocity error |d(u,v)_i| / max(|(u,v)_i|, rms |(u,v)|) against a reference."""
    u, v, ur, vr = (np.asarray(a, dtype=np.float64) for a in (u, v, ur, vr))
    mag = np.hypot(ur, vr)
    rms = np.sqrt(np.mean(mag * mag)) if mag.size else 0.0
    scale = np.maximum(mag, rms)
    scale = np.where(scale > 0, scale, 1.0)
    return np.hypot(u - ur, v - vr) / scale


def position_error(x, y, xr, yr) -> float:
    """max |d(x,y)_i| / max(1, max |(x,y)|)."""
    d = np.hypot(np.asarray(x) - xr, np.asarray(y) - yr)
    return float(d.max() / max(1.0, float(np.hypot(xr, yr).max()))) if d.size else 0.0
