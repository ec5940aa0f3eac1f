"""The FP32-compensated precision form (PV_PRECISION_FP32C) against the FP64 oracle.

What bounds its error. Every far term is evaluated in FP32 from double-float displacements, so it
carries a relative error of a few FP32 ulp: rcp.approx (one ulp) and about four roundings, below
2^-22 ~ 2.4e-7 of the term. The terms of one velocity have random signs and the FP32 partial sums
are promoted into FP64 every 64 sources, so these errors add like a random walk, as the terms do:
the per-vortex error normalised by max(|(u,v)_i|, rms |(u,v)|) has an rms below 2^-22 whatever N.
Its maximum is set by the largest FP32 terms, those of the closest pairs: the near field (terms
within the near-field radius evaluated in FP64: periodic pairs, disk pairs and disk wall images)
takes them out, which caps the maximum near 2^-20 ~ 9.5e-7 at the default radius. The plane has no
near field, and its maximum stays near 2^-18 ~ 3.8e-6. These are the bounds asserted here; an FP32
term cannot reach the 1e-9 of an FP64 evaluation, and the near-field radius trades the maximum
error against speed (bench.py --fp32c-curve)."""
import numpy as np
import pytest

import pointvortex_b200 as pv
from conftest import golden, normalized_error
from oracle.pyoracle import Geometry
from pointvortex_b200 import ics

pytestmark = pytest.mark.gpu

RMS_BOUND = 2.0 ** -22
MAX_BOUND = {"infinite": 2.0 ** -18, "periodic": 2.0 ** -20, "disk": 2.0 ** -20}


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


def errors(f, ur, vr):
    err = normalized_error(f.x, f.y, ur, vr)
    return float(err.max()), float(np.sqrt(np.mean(err ** 2)))


GEO = {"infinite": Geometry("infinite"),
       "periodic": Geometry("periodic", box_length_x=2 * np.pi, box_length_y=2 * np.pi),
       "disk": Geometry("disk", disk_radius=1.0)}


@pytest.mark.parametrize("boundary", ["infinite", "periodic", "disk"])
@pytest.mark.parametrize("n", [3, 257, 2000])
def test_fp32c_error_against_fp64_oracle(port, boundary, n):
    x, y, g = state(boundary, n, 40 + n)
    f = kernel(boundary).evaluate(x, y, g)
    ur, vr = port.evaluate(GEO[boundary], x, y, g)
    mx, rms = errors(f, ur, vr)
    print(f"{boundary} n={n}: fp32c error max {mx:.2e} rms {rms:.2e}")
    assert mx <= MAX_BOUND[boundary] and rms <= RMS_BOUND


def test_fp32c_workload_fixtures():
    for name, boundary in [("workload_infinite_n1024.npz", "infinite"),
                           ("workload_periodic_n4096.npz", "periodic"),
                           ("workload_disk_n16384.npz", "disk")]:
        d = golden(name)
        f = kernel(boundary).evaluate(d["x"], d["y"], d["g"])
        k = d["u"].size
        err = normalized_error(f.x[:k], f.y[:k], d["u"], d["v"])
        print(f"{name}: fp32c error max {err.max():.2e} rms {np.sqrt(np.mean(err**2)):.2e}")
        assert err.max() <= MAX_BOUND[boundary]


@pytest.mark.parametrize("boundary", ["periodic", "disk"])
def test_near_field_lowers_the_maximum_error(port, boundary):
    """The same state without a near field (radius 0), at the default radius, and at a radius
    whose lists overflow (every target then evaluated whole in FP64): the maximum error falls, and
    in the last case the result is FP64's."""
    n = 4096 if boundary == "periodic" else 6000
    x, y, g = state(boundary, n, 77)
    ur, vr = port.evaluate(GEO[boundary], x, y, g)
    k = kernel(boundary)
    k.uploadDeviceState(pv.VortexSystem(x, y, g))
    default = k.nearField
    assert default > 0
    k.setNearField(0.0)
    mx0, _ = errors(k.evaluateDeviceState(), ur, vr)
    k.setNearField(-1.0)
    assert k.nearField == default
    mx1, rms1 = errors(k.evaluateDeviceState(), ur, vr)
    k.setNearField(8 * default)
    mx2, _ = errors(k.evaluateDeviceState(), ur, vr)
    print(f"{boundary}: max error without near field {mx0:.2e}, default radius {mx1:.2e} "
          f"(rms {rms1:.2e}), overflowing radius {mx2:.2e}")
    assert mx1 < mx0 and mx1 <= MAX_BOUND[boundary] and rms1 <= RMS_BOUND
    assert mx2 <= 1e-12


def test_near_field_evaluation_is_deterministic():
    x, y, g = state("periodic", 4096, 78)
    k = kernel("periodic")
    k.uploadDeviceState(pv.VortexSystem(x, y, g))
    a = k.evaluateDeviceState()
    b = k.evaluateDeviceState()
    assert np.array_equal(a.x, b.x) and np.array_equal(a.y, b.y)
    xd, yd, gd = state("disk", 3000, 79)
    kd = kernel("disk")
    c = kd.evaluate(xd, yd, gd)
    d = kd.evaluate(xd, yd, gd)
    assert np.array_equal(c.x, d.x) and np.array_equal(c.y, d.y)


def test_fp32c_coincident_and_errors_like_fp64():
    x = np.array([0.1, -0.2, 0.1])
    y = np.array([0.0, 0.1, 0.0])
    g = np.array([1.0, -1.0, 1.0])
    with pytest.raises(RuntimeError, match="coincident"):
        kernel("infinite").evaluate(x, y, g)
    # in the periodic box and the disk a coincident pair is in the near field: the FP64 pass
    # meets it and the slow path reports the reference's error
    xp, yp, gp = state("periodic", 64, 80)
    xp[3], yp[3] = xp[7], yp[7]
    with pytest.raises(RuntimeError, match="coincident periodic vortices"):
        kernel("periodic").evaluate(xp, yp, gp)
    xd, yd, gd = state("disk", 64, 81)
    xd[3], yd[3] = xd[7], yd[7]
    with pytest.raises(RuntimeError, match="coincident vortices in disk"):
        kernel("disk").evaluate(xd, yd, gd)


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
    ur, vr = reference.evaluate(GEO["periodic"], x, y, g)
    mx, rms = errors(f, ur, vr)
    print(f"symmetric periodic n={n}: fp32c error max {mx:.2e} rms {rms:.2e}")
    assert mx <= MAX_BOUND["periodic"] and rms <= RMS_BOUND
    ordered = k.evaluate(x, y, g)   # host arrays: the ordered FP32C kernel
    assert normalized_error(f.x, f.y, ordered.x, ordered.y).max() <= MAX_BOUND["periodic"]
