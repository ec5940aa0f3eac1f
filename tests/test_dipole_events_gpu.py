"""Dipole events on the device state (DeviceDipoleManager / pv_dipole_process) against three
consecutive DipoleManager::process calls of the reference (golden fixtures): population, order,
positions, circulations, counts and the generator's text state all bit-exact; the velocity of
the compacted device state against the oracle; restore from a checkpointed state; errors."""
import numpy as np
import pytest

import pointvortex_b200 as pv
from golden.make_golden import dipole_event_geometry

pytestmark = pytest.mark.gpu

CASES = [(b, m) for b in ("periodic", "disk") for m in (0, 1, 2)]
MODES = {0: "none", 1: "independent", 2: "paired"}


def kernel_for(boundary):
    if boundary == "periodic":
        return pv.PeriodicBoxKernel(2 * np.pi, 2 * np.pi, 8)
    return pv.DiskKernel(1.0)


def manager(k, mode, state=None):
    return pv.DeviceDipoleManager(k, removal=True, distance=0.02, reinjection=MODES[mode],
                                  random_seed=99, state=state)


@pytest.mark.parametrize("boundary,mode", CASES)
def test_device_events_match_reference(boundary, mode):
    from conftest import golden
    d = golden(f"dipole_events_{boundary}_{mode}.npz")
    k = kernel_for(boundary)
    k.uploadDeviceState(pv.VortexSystem(d["x"], d["y"], d["g"]))
    dm = manager(k, mode)
    for call in range(3):
        events = dm.process()
        s = k.downloadDeviceSystem()
        assert events == int(d[f"events{call}"][0]), call
        assert np.array_equal(s.x, d[f"x{call}"]) and np.array_equal(s.y, d[f"y{call}"]), call
        assert np.array_equal(s.circulation, d[f"g{call}"]), call
        st = dm.state()
        assert (st.removedPairs, st.reinjectedPairs) == tuple(int(c) for c in d[f"counts{call}"])
        assert st.randomEngineState == str(d[f"engine{call}"])


@pytest.mark.parametrize("boundary,mode", [("periodic", 2), ("disk", 1)])
def test_velocity_of_compacted_state(port, boundary, mode):
    """The compaction moves the scaled circulations with the positions: the device-state
    velocity after the events equals the oracle's velocity of the reference's new state."""
    from conftest import golden, normalized_error
    d = golden(f"dipole_events_{boundary}_{mode}.npz")
    geo = dipole_event_geometry(boundary, mode)
    k = kernel_for(boundary)
    k.uploadDeviceState(pv.VortexSystem(d["x"], d["y"], d["g"]))
    manager(k, mode).process()
    vel = k.evaluateDeviceState()
    u, v = port.evaluate(geo, d["x0"], d["y0"], d["g0"])
    assert normalized_error(vel.x, vel.y, u, v).max() <= 1e-12


@pytest.mark.parametrize("boundary,mode", [("periodic", 1), ("disk", 1)])
def test_restore_from_checkpointed_state(boundary, mode):
    """A manager restored from the state after call 0 (DipoleManager(params, state)) continues
    exactly as the uninterrupted reference manager did."""
    from conftest import golden
    d = golden(f"dipole_events_{boundary}_{mode}.npz")
    counts = [int(c) for c in d["counts0"]]
    state = pv.DipoleEventState(counts[0], counts[1], str(d["engine0"]))
    k = kernel_for(boundary)
    k.uploadDeviceState(pv.VortexSystem(d["x0"], d["y0"], d["g0"]))
    dm = manager(k, mode, state)
    for call in (1, 2):
        assert dm.process() == int(d[f"events{call}"][0])
        s = k.downloadDeviceSystem()
        assert np.array_equal(s.x, d[f"x{call}"]) and np.array_equal(s.y, d[f"y{call}"])
        assert dm.state().randomEngineState == str(d[f"engine{call}"])


def test_no_candidates_leaves_state_and_generator_alone():
    from conftest import golden
    d = golden("dipole_events_periodic_1.npz")
    k = kernel_for("periodic")
    k.uploadDeviceState(pv.VortexSystem(d["x0"], d["y0"], d["g0"]))
    dm = manager(k, 1)
    before = dm.state()
    assert dm.process() == 0
    s = k.downloadDeviceSystem()
    assert np.array_equal(s.x, d["x0"]) and dm.state() == before


def test_errors():
    k = pv.InfinitePlaneKernel(0.0)
    with pytest.raises(ValueError, match="only for periodic and disk"):
        pv.DeviceDipoleManager(k, reinjection="paired")
    with pytest.raises(ValueError, match="requires dipoleRemoval"):
        pv.DeviceDipoleManager(kernel_for("disk"), removal=False, reinjection="independent")
    with pytest.raises(ValueError, match="must be positive"):
        pv.DeviceDipoleManager(k, distance=0.0)
    dm = pv.DeviceDipoleManager(k)
    with pytest.raises(pv.LogicError, match="not been uploaded"):
        dm.process()
    with pytest.raises(RuntimeError, match="invalid random-generator state"):
        pv.DeviceDipoleManager(k, state=pv.DipoleEventState(0, 0, "1 2 three"))


def test_disabled_removal_is_a_no_op():
    from conftest import golden
    d = golden("dipole_events_disk_0.npz")
    k = kernel_for("disk")
    k.uploadDeviceState(pv.VortexSystem(d["x"], d["y"], d["g"]))
    dm = pv.DeviceDipoleManager(k, removal=False, distance=0.02)
    assert dm.process() == 0 and k.stateSize() == d["x"].size


@pytest.mark.parametrize("planted", [True, False])
def test_scan_fused_into_the_step(planted):
    """With removal configured, each DOPRI5 attempt also scans its accepted state; process()
    after the step must give what a fresh scan of that state gives (events, population, order)."""
    from conftest import golden
    d = golden("dipole_events_periodic_0.npz")
    x, y, g = (d["x"], d["y"], d["g"]) if planted else (d["x0"], d["y0"], d["g0"])
    fused = kernel_for("periodic")
    fused.uploadDeviceState(pv.VortexSystem(x, y, g))
    dm = manager(fused, 0)
    fused.deviceDopri5Step(1e-7, 1e-12, 1e-9, 1e-12, 0.1)
    stepped = fused.downloadDeviceSystem()
    events = dm.process()
    after = fused.downloadDeviceSystem()
    fresh = kernel_for("periodic")
    fresh.uploadDeviceState(stepped)
    want = manager(fresh, 0).process()
    expect = fresh.downloadDeviceSystem()
    assert events == want and (events > 0) == planted
    assert np.array_equal(after.x, expect.x) and np.array_equal(after.circulation, expect.circulation)
