"""The exits of the bounded device waits, driven on purpose (pv_set_wait_limits).

Every device-side wait of the library is bounded: a velocity launch's wait for its tile copies
(mbarrier), and the grid barrier of the cooperative RK4 steps. A wait that runs out sets the status
word to ST_TIMEOUT and the kernel returns; the host maps it to the runtime error "a bounded device
wait timed out". The waits here run out because the test shortens their limit to zero polls -- a
wait that gives up at once, with nothing left pending on the device: a velocity tile first waits,
with the default bound, for its copies still in flight, and a broken grid barrier is seen by every
CTA. Nothing faults, traps or hangs. Each test then checks that the state is consistent (unchanged
for a single step, a whole number of completed steps for a multi-step advance) and that the same
context works again once the default limits are back."""
import numpy as np
import pytest

import pointvortex_b200 as pv
from conftest import normalized_error, position_error  # noqa: F401
from oracle.pyoracle import Geometry
from pointvortex_b200 import ics

pytestmark = pytest.mark.gpu

TIMEOUT = "a bounded device wait timed out"


def download(k, n, g):
    s = pv.VortexSystem(np.zeros(n), np.zeros(n), g)
    k.downloadDeviceState(s)
    return s.x.copy(), s.y.copy()


def test_velocity_tile_wait_runs_out(port):
    x, y, g = ics.periodic_box(600, 31, 2.0)
    k = pv.PeriodicBoxKernel(2.0, 2.0, 8)
    k.setWaitLimits(copy_polls=0)
    for _ in range(2):
        with pytest.raises(RuntimeError, match=TIMEOUT):
            k.evaluate(x, y, g)
    k.setWaitLimits()
    f = k.evaluate(x, y, g)
    ur, vr = port.evaluate(Geometry("periodic", box_length_x=2.0, box_length_y=2.0), x, y, g)
    assert normalized_error(f.x, f.y, ur, vr).max() <= 1e-12


def test_velocity_timeout_inside_a_step_leaves_the_state(port):
    # N > 2048: the step is the launch sequence (tiled velocity kernel + stage kernels)
    x, y, g = ics.infinite_plane(3000, 32)
    k = pv.InfinitePlaneKernel(0.0)
    k.uploadDeviceState(pv.VortexSystem(x, y, g))
    k.setWaitLimits(copy_polls=0)
    with pytest.raises(RuntimeError, match=TIMEOUT):
        k.deviceRk4Step(1e-3)
    sx, sy = download(k, x.size, g)
    assert np.array_equal(sx, x) and np.array_equal(sy, y)
    with pytest.raises(RuntimeError, match=TIMEOUT):
        k.deviceDopri5Step(1e-3, 1e-10, 1e-8, 1e-12, 0.1)
    sx, sy = download(k, x.size, g)
    assert np.array_equal(sx, x) and np.array_equal(sy, y)
    k.setWaitLimits()
    k.deviceRk4Step(1e-3)
    sx, sy = download(k, x.size, g)
    # the same step on a context whose waits never ran out: bit for bit
    fresh = pv.InfinitePlaneKernel(0.0)
    fresh.uploadDeviceState(pv.VortexSystem(x, y, g))
    fresh.deviceRk4Step(1e-3)
    fx, fy = download(fresh, x.size, g)
    assert np.array_equal(sx, fx) and np.array_equal(sy, fy)
    # and the reference's step, within the teacher-forced tolerance (1e-12 dt max|u|)
    u, v = port.evaluate(Geometry("infinite"), x, y, g)
    rx, ry = port.stepper(Geometry("infinite"), x.size).rk4_step(x, y, g, 1e-3)
    tol = 1e-12 * 1e-3 * float(np.hypot(u, v).max())
    assert float(np.max(np.hypot(sx - rx, sy - ry))) <= tol


def plain_steps(x, y, g, steps):
    """The states after 1..steps RK4 steps (dt 1e-3) on a context whose waits keep their
    defaults."""
    k = pv.InfinitePlaneKernel(0.0)
    k.uploadDeviceState(pv.VortexSystem(x, y, g))
    out = [(x.copy(), y.copy())]
    for _ in range(steps):
        k.deviceRk4Step(1e-3)
        out.append(download(k, x.size, g))
    k.close()
    return out


def test_cooperative_barrier_timeout_is_agreed(port):
    # N <= 2048 FP64: RK4 steps run as one cooperative launch with a grid barrier per stage
    geo = Geometry("infinite")
    x, y, g = ics.infinite_plane(1024, 33)
    k = pv.InfinitePlaneKernel(0.0)
    rx, ry = plain_steps(x, y, g, 1)[1]
    u, v = port.evaluate(geo, x, y, g)
    ox, oy = port.stepper(geo, x.size).rk4_step(x, y, g, 1e-3)
    # the undisturbed GPU step against the reference's: the teacher-forced tolerance
    assert float(np.max(np.hypot(rx - ox, ry - oy))) <= 1e-12 * 1e-3 * float(np.hypot(u, v).max())
    timeouts = 0
    for _ in range(8):
        k.uploadDeviceState(pv.VortexSystem(x, y, g))
        k.setWaitLimits(barrier_polls=0)
        try:
            k.deviceRk4Step(1e-3)
        except RuntimeError as exc:
            assert TIMEOUT in str(exc)
            timeouts += 1
            sx, sy = download(k, x.size, g)
            assert np.array_equal(sx, x) and np.array_equal(sy, y)
        else:  # every CTA arrived before any gave up: an ordinary step, bit for bit
            sx, sy = download(k, x.size, g)
            assert np.array_equal(sx, rx) and np.array_equal(sy, ry)
    # a barrier that gives up at once breaks unless all 148 CTAs arrive within the same instant
    assert timeouts >= 1
    k.setWaitLimits()
    k.uploadDeviceState(pv.VortexSystem(x, y, g))
    k.deviceRk4Step(1e-3)
    sx, sy = download(k, x.size, g)
    assert np.array_equal(sx, rx) and np.array_equal(sy, ry)


def test_cooperative_advance_timeout_stops_at_a_whole_step(port):
    x, y, g = ics.infinite_plane(1024, 34)
    steps = 4
    states = plain_steps(x, y, g, steps)  # the cooperative launch is bit for bit the same
    k = pv.InfinitePlaneKernel(0.0)
    for _ in range(4):
        k.uploadDeviceState(pv.VortexSystem(x, y, g))
        k.setWaitLimits(barrier_polls=0)
        try:
            k.rk4Advance(1e-3, steps)
            done = steps
        except RuntimeError as exc:
            assert TIMEOUT in str(exc)
            done = None
        sx, sy = download(k, x.size, g)
        # the state is that of a whole number of steps, bit for bit
        matches = [i for i, (a, b) in enumerate(states)
                   if np.array_equal(sx, a) and np.array_equal(sy, b)]
        assert len(matches) == 1, [position_error(sx, sy, a, b) for a, b in states]
        best = matches[0]
        if done is not None:
            assert best == steps
        else:
            assert best < steps
    k.setWaitLimits()
