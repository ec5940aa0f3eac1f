"""The FP32-compensated precision form (PV_PRECISION_FP32C) against the FP64 oracle. The error it
reaches is a property of FP32 pair terms (a few ulp each, ~1e-7 relative); the bounds below are
the measured errors with a margin, per geometry, normalised as the FP64 parity tests are."""
import numpy as np
import pytest

import pointvortex_b200 as pv
from conftest import golden, normalized_error
from oracle.pyoracle import Geometry
from pointvortex_b200 import ics

pytestmark = pytest.mark.gpu

# per-vortex |d(u,v)_i| / max(|(u,v)_i|, rms|(u,v)|): max and rms bounds, measured on B200 with a
# margin (periodic N = 2000: max 8.9e-6, rms 3.3e-7; the plane and the disk stay below 2e-6 / 2e-7)
BOUNDS = {"infinite": (2e-6, 2e-7), "periodic": (2e-5, 1e-6), "disk": (2e-6, 2e-7)}


def kernel(boundary, precision=1):
    if boundary == "infinite":
        return pv.InfinitePlaneKernel(0.0, precision=precision)
    if boundary == "periodic":
        return pv.PeriodicBoxKernel(2 * np.pi, 2 * np.pi, 8, precision=precision)
    return pv.DiskKernel(1.0, precision=precision)


def state(boundary, n, seed):
    if boundary == "periodic":
        return ics.periodic_box(n + n % 2, seed)
    if boundary == "disk":
        return ics.disk(n, seed, 1.0, 0.95)
    return ics.infinite_plane(n, seed)


@pytest.mark.parametrize("boundary", ["infinite", "periodic", "disk"])
@pytest.mark.parametrize("n", [3, 257, 2000])
def test_fp32c_error_against_fp64_oracle(port, boundary, n):
    x, y, g = state(boundary, n, 40 + n)
    f = kernel(boundary).evaluate(x, y, g)
    geo = Geometry(boundary, box_length_x=2 * np.pi, box_length_y=2 * np.pi, disk_radius=1.0)
    ur, vr = port.evaluate(geo, x, y, g)
    err = normalized_error(f.x, f.y, ur, vr)
    mx, rms = BOUNDS[boundary]
    print(f"{boundary} n={n}: fp32c error max {err.max():.2e} rms {np.sqrt(np.mean(err**2)):.2e}")
    assert err.max() <= mx and np.sqrt(np.mean(err ** 2)) <= rms


def test_fp32c_workload_fixtures():
    for name, boundary in [("workload_infinite_n1024.npz", "infinite"),
                           ("workload_periodic_n4096.npz", "periodic"),
                           ("workload_disk_n16384.npz", "disk")]:
        d = golden(name)
        f = kernel(boundary).evaluate(d["x"], d["y"], d["g"])
        k = d["u"].size
        err = normalized_error(f.x[:k], f.y[:k], d["u"], d["v"])
        print(f"{name}: fp32c error max {err.max():.2e} rms {np.sqrt(np.mean(err**2)):.2e}")
        assert err.max() <= BOUNDS[boundary][0]


def test_fp32c_coincident_and_errors_like_fp64():
    x = np.array([0.1, -0.2, 0.1])
    y = np.array([0.0, 0.1, 0.0])
    g = np.array([1.0, -1.0, 1.0])
    with pytest.raises(RuntimeError, match="coincident"):
        kernel("infinite").evaluate(x, y, g)


def test_fp32c_steps_track_fp64():
    x, y, g = state("disk", 800, 3)
    ks = [kernel("disk", p) for p in (0, 1)]
    out = []
    for k in ks:
        k.uploadDeviceState(pv.VortexSystem(x, y, g))
        for _ in range(5):
            k.deviceRk4Step(1e-4)
        s = pv.VortexSystem(x.copy(), y.copy(), g)
        k.downloadDeviceState(s)
        out.append(s)
    # five steps of 1e-4 with Gaussian circulations (speeds up to ~1e3): FP32-level velocity
    # differences move the vortices by ~1e-7 at most
    assert np.max(np.hypot(out[0].x - out[1].x, out[0].y - out[1].y)) < 1e-6


@pytest.mark.parametrize("n", [2082, 4096])
def test_fp32c_symmetric_periodic_against_fp64_oracle(reference, n):
    """From N = 2048 the compensated periodic evaluation of the device state runs once per
    unordered pair (its FP32 terms are exactly odd as well); same bounds as the ordered form."""
    x, y, g = state("periodic", n, 70 + n)
    k = kernel("periodic")
    k.uploadDeviceState(pv.VortexSystem(x, y, g))
    assert k.statePlan()["symmetric"]
    f = k.evaluateDeviceState()
    geo = Geometry("periodic", box_length_x=2 * np.pi, box_length_y=2 * np.pi)
    ur, vr = reference.evaluate(geo, x, y, g)
    err = normalized_error(f.x, f.y, ur, vr)
    mx, rms = BOUNDS["periodic"]
    print(f"symmetric periodic n={n}: fp32c error max {err.max():.2e} "
          f"rms {np.sqrt(np.mean(err**2)):.2e}")
    assert err.max() <= mx and np.sqrt(np.mean(err ** 2)) <= rms
    ordered = k.evaluate(x, y, g)   # host arrays: the ordered FP32C kernel
    assert normalized_error(f.x, f.y, ordered.x, ordered.y).max() <= mx
