"""Device-resident RK4 / DOPRI5 stepping against the oracle's RungeKuttaIntegrator.

The workloads are chaotic (a 1-ulp change grows to O(0.1) in 20 RK4 steps of the N=1024 case), so
trajectories are compared teacher-forced: from the same state, one GPU step against one oracle
step. The combination arithmetic is the reference's, rounded operation by operation, so the step
error is the velocity difference times dt."""
import dataclasses

import numpy as np
import pytest

import pointvortex_b200 as pv
from conftest import golden, position_error
from gpu_impl import GpuStepper, make_kernel
from oracle.pyoracle import Geometry
from pointvortex_b200 import ics

pytestmark = pytest.mark.gpu

GEOS = {
    "infinite": Geometry("infinite"),
    "periodic": Geometry("periodic", box_length_x=2.0, box_length_y=2.0),
    "disk": Geometry("disk", disk_radius=1.0),
}


def state(name, n, seed):
    if name == "periodic":
        return ics.periodic_box(n, seed, 2.0)
    if name == "disk":
        return ics.disk(n, seed, 1.0, 0.8, gaussian=False)
    return ics.infinite_plane(n, seed)


@pytest.mark.parametrize("name", sorted(GEOS))
def test_rk4_teacher_forced(port, name):
    geo = GEOS[name]
    x, y, g = state(name, 300, 21)
    ref = port.stepper(geo, x.size)
    for k in range(5):
        gpu = GpuStepper(geo)
        gx, gy = gpu.rk4_step(x, y, g, 1e-3)
        rx, ry = ref.rk4_step(x, y, g, 1e-3)
        assert position_error(gx, gy, rx, ry) <= step_tolerance(port, geo, x, y, g, 1e-3)
        x, y = rx, ry


@pytest.mark.parametrize("tag", ["infinite", "infinite_core", "periodic", "periodic_m3", "disk"])
def test_small_fixture_steps(tag):
    geos = {"infinite": Geometry("infinite"), "infinite_core": Geometry("infinite", core_radius=0.05),
            "periodic": GEOS["periodic"],
            "periodic_m3": Geometry("periodic", box_length_x=2.0, box_length_y=2.0, image_layers=3),
            "disk": GEOS["disk"]}
    geo = geos[tag]
    d = golden(f"small_{tag}.npz")
    g = d["g"]
    for k in range(3):
        gx, gy = GpuStepper(geo).rk4_step(d["rk_x"][k], d["rk_y"][k], g, 1e-3)
        assert position_error(gx, gy, d["rk_x"][k + 1], d["rk_y"][k + 1]) <= 1e-14
    st = GpuStepper(geo)
    cx, cy, dt = d["x"], d["y"], 1e-3
    for k in range(3):
        cx, cy, r = st.dopri5_step(cx, cy, g, dt)
        rr = d["dp_r"][k]
        assert r[3] == rr[3]
        # without rejections the accepted step is the requested one; after rejections it carries
        # the error estimate's relative precision (~1e-11) through pow(err, -0.2)
        assert r[0] == rr[0] if rr[3] == 0 else abs(r[0] - rr[0]) <= 1e-9 * rr[0]
        assert abs(r[1] - rr[1]) <= 1e-9 * rr[1]
        assert abs(r[2] - rr[2]) <= 1e-6 * max(rr[2], 1e-3)
        assert position_error(cx, cy, d["dp_x"][k + 1], d["dp_y"][k + 1]) <= 1e-13
        # continue from the reference's state (teacher forcing), keeping FSAL as the reference does
        dt = rr[1]


def step_tolerance(port, geo, x, y, g, dt):
    """A velocity difference of 1e-12 (relative to the largest speed) moves a vortex by at most
    1e-12 * dt * max|u| per step; close pairs make max|u| large (~300 in the N=1024 workload)."""
    u, v = port.evaluate(geo, x, y, g)
    return max(1e-12 * dt * float(np.hypot(u, v).max()), 1e-15)


def test_workload_rk4_teacher_forced(port):
    d = golden("workload_infinite_n1024.npz")
    geo = Geometry("infinite")
    for k in range(5):
        gx, gy = GpuStepper(geo).rk4_step(d["rk_x"][k], d["rk_y"][k], d["g"], 1e-3)
        tol = step_tolerance(port, geo, d["rk_x"][k], d["rk_y"][k], d["g"], 1e-3)
        assert position_error(gx, gy, d["rk_x"][k + 1], d["rk_y"][k + 1]) <= tol


@pytest.mark.parametrize("name", sorted(GEOS))
def test_dopri_sequence_against_oracle(port, name):
    geo = dataclasses.replace(GEOS[name], relative_tolerance=1e-9, absolute_tolerance=1e-12)
    x, y, g = state(name, 200, 31)
    ref = port.stepper(geo, x.size)
    gpu = GpuStepper(geo)
    rx, ry, gx, gy = x, y, x, y
    dt = 1e-3
    for _ in range(4):
        rx2, ry2, rr = ref.dopri5_step(rx, ry, g, dt)
        # teacher forcing: the GPU steps from the oracle's state; the upload only happens when the
        # state differs from what the GPU produced last step
        gx, gy, gr = gpu.dopri5_step(rx, ry, g, dt)
        assert gr[3] == rr[3]
        assert gr[0] == rr[0] if rr[3] == 0 else abs(gr[0] - rr[0]) <= 1e-9 * rr[0]
        assert position_error(gx, gy, rx2, ry2) <= 1e-13
        rx, ry, dt = rx2, ry2, rr[1]


def test_rk4_advance_equals_steps():
    geo = GEOS["periodic"]
    x, y, g = state("periodic", 500, 41)
    a = make_kernel(geo)
    b = make_kernel(geo)
    a.uploadDeviceState(pv.VortexSystem(x, y, g))
    b.uploadDeviceState(pv.VortexSystem(x, y, g))
    for _ in range(6):
        a.deviceRk4Step(1e-3)
    b.rk4Advance(1e-3, 6)
    sa = pv.VortexSystem(x.copy(), y.copy(), g)
    sb = pv.VortexSystem(x.copy(), y.copy(), g)
    a.downloadDeviceState(sa)
    b.downloadDeviceState(sb)
    assert np.array_equal(sa.x, sb.x) and np.array_equal(sa.y, sb.y)
    assert a.evaluationCount == b.evaluationCount == 24


def test_step_failure_leaves_state_unchanged(port):
    """A disk vortex pushed through the wall: the reference throws "vortex lies on or outside the
    disk" at the next evaluation; the device state keeps the last good positions."""
    geo = GEOS["disk"]
    x = np.array([0.9999, -0.2])
    y = np.array([0.0, 0.0])
    g = np.array([1.0, 50.0])
    k = make_kernel(geo)
    s = pv.VortexSystem(x, y, g)
    k.uploadDeviceState(s)
    with pytest.raises(ValueError) as gpu_err:
        for _ in range(50):
            k.deviceRk4Step(1e-2)
    st = port.stepper(geo, 2)
    with pytest.raises(ValueError) as ref_err:
        cx, cy = x, y
        for _ in range(50):
            cx, cy = st.rk4_step(cx, cy, g, 1e-2)
    assert str(gpu_err.value) == str(ref_err.value) == "vortex lies on or outside the disk"
    after = pv.VortexSystem(x.copy(), y.copy(), g)
    k.downloadDeviceState(after)
    assert np.all(after.x ** 2 + after.y ** 2 < 1.0)


def test_hooks_require_upload():
    k = make_kernel(GEOS["infinite"])
    with pytest.raises(pv.LogicError):
        k.deviceRk4Step(1e-3)
    k.uploadDeviceState(pv.VortexSystem([0.0, 1.0], [0.0, 0.0], [1.0, 1.0]))
    with pytest.raises(RuntimeError, match="populations differ"):
        k.downloadDeviceState(pv.VortexSystem([0.0], [0.0], [1.0]))


def test_dopri_rejection_cap(port):
    """An impossible tolerance makes the reference give up after 32 rejections."""
    geo = Geometry("infinite", absolute_tolerance=1e-300, relative_tolerance=0.0,
                   minimum_time_step=1e-300, maximum_time_step=1.0)
    x, y, g = ics.infinite_plane(50, 3)
    with pytest.raises(RuntimeError) as ge:
        GpuStepper(geo).dopri5_step(x, y, g, 0.1)
    with pytest.raises(RuntimeError) as re_:
        port.stepper(geo, x.size).dopri5_step(x, y, g, 0.1)
    assert str(ge.value) == str(re_.value)


def test_empty_population():
    k = make_kernel(GEOS["infinite"])
    k.uploadDeviceState(pv.VortexSystem([], [], []))
    k.deviceRk4Step(1e-3)
    r = k.deviceDopri5Step(1e-3, 1e-10, 1e-8, 1e-12, 0.1)
    assert r.acceptedTimeStep == 1e-3 and r.suggestedTimeStep == 5e-3 and r.rejectedSteps == 0


def test_dopri_graph_replay_equals_launches_and_profiling():
    """The FSAL attempt is replayed as a captured CUDA graph (with per-launch event nodes when
    profiling): steps with profiling on and off give identical states and step results."""
    import pointvortex_b200 as pv
    from pointvortex_b200 import ics
    x, y, g = ics.periodic_box(2100, 31)
    out = []
    for profiling in (False, True):
        k = pv.PeriodicBoxKernel(2 * np.pi, 2 * np.pi, 8)
        k.setProfiling(profiling)
        k.uploadDeviceState(pv.VortexSystem(x, y, g))
        dt, results = 1e-4, []
        for _ in range(6):
            r = k.deviceDopri5Step(dt, 1e-12, 1e-9, 1e-12, 0.1)
            results.append((r.acceptedTimeStep, r.rejectedSteps))
            dt = r.suggestedTimeStep
        s = k.downloadDeviceSystem()
        stats = k.kernelStats()
        out.append((results, s.x, s.y, stats))
    (r0, x0, y0, _), (r1, x1, y1, st1) = out
    assert r0 == r1 and np.array_equal(x0, x1) and np.array_equal(y0, y1)
    launches, timed, ms = st1["velocity"]
    assert launches == timed and ms > 0  # every replayed launch was timed by its graph events


@pytest.mark.parametrize("name", sorted(GEOS))
@pytest.mark.parametrize("n", [300, 1024, 2048])
def test_rk4_cooperative_steps_equal_the_launch_sequence(name, n):
    """Small FP64 populations take whole RK4 steps in one cooperative launch; with per-launch
    profiling on, the same steps run as the launch sequence. Both give the same state bit for
    bit, through rk4Advance and through single steps, or stop with the same error (a disk vortex
    of a close pair can leave the disk) at the same state."""
    geo = GEOS[name]
    x, y, g = state(name, n, 70 + n)
    ks = []
    for profiling in (False, True):
        k = make_kernel(geo)
        k.uploadDeviceState(pv.VortexSystem(x, y, g))
        k.setProfiling(profiling)
        k.resetKernelStats()
        error = None
        try:
            k.rk4Advance(5e-4, 7)
            for _ in range(3):
                k.deviceRk4Step(5e-4)
        except ValueError as exc:
            error = str(exc)
        out = pv.VortexSystem(x.copy(), y.copy(), g)
        k.downloadDeviceState(out)
        ks.append((k, out, error))
    (fast, a, ea), (_, b, eb) = ks
    assert ea == eb
    assert np.array_equal(a.x, b.x) and np.array_equal(a.y, b.y)
    if ea is None:
        assert fast.evaluationCount == 40
        if n == 1024:  # one launch for the 7 steps and one per single step
            assert fast.kernelStats()["velocity"][0] == 4


def test_rk4_cooperative_failure_keeps_the_last_state(port):
    """A disk vortex pushed through the wall inside rk4Advance: the reference's error, and the
    state after the last good step, as with the launch sequence."""
    geo = GEOS["disk"]
    x = np.array([0.9999, -0.2])
    y = np.array([0.0, 0.0])
    g = np.array([1.0, 50.0])
    outs = []
    for profiling in (False, True):
        k = make_kernel(geo)
        k.uploadDeviceState(pv.VortexSystem(x, y, g))
        k.setProfiling(profiling)
        with pytest.raises(ValueError, match="vortex lies on or outside the disk"):
            k.rk4Advance(1e-2, 50)
        out = pv.VortexSystem(x.copy(), y.copy(), g)
        k.downloadDeviceState(out)
        outs.append(out)
    assert np.array_equal(outs[0].x, outs[1].x) and np.array_equal(outs[0].y, outs[1].y)
    assert np.all(outs[0].x ** 2 + outs[0].y ** 2 < 1.0)
