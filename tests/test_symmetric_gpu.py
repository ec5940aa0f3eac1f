"""The periodic box and the infinite plane evaluated once per unordered pair (the device-state
path from N = 2048 and N = 16384 up): against the oracle and against the ordered-pair kernel, on
ragged populations, with more than one sub-block per block, deterministic, and with the
reference's errors."""
import numpy as np
import pytest

import pointvortex_b200 as pv
from conftest import golden, normalized_error
from oracle.pyoracle import Geometry
from pointvortex_b200 import _lib, ics

pytestmark = pytest.mark.gpu

L = 2 * np.pi


def kernel_with(x, y, g, length=L, layers=8):
    k = pv.PeriodicBoxKernel(length, length, layers)
    k.uploadDeviceState(pv.VortexSystem(x, y, g))
    return k


@pytest.mark.parametrize("n,layers", [(2082, 8), (3000, 3), (4096, 8)])
def test_symmetric_matches_oracle(reference, n, layers):
    x, y, g = ics.periodic_box(n, 40 + n, L)
    k = kernel_with(x, y, g, layers=layers)
    assert k.statePlan()["symmetric"]
    vel = k.evaluateDeviceState()
    geo = Geometry("periodic", box_length_x=L, box_length_y=L, image_layers=layers)
    u, v = reference.evaluate(geo, x, y, g)
    assert normalized_error(vel.x, vel.y, u, v).max() <= 1e-12


def test_symmetric_on_the_workload_fixture():
    d = golden("workload_periodic_n4096.npz")
    k = kernel_with(d["x"], d["y"], d["g"])
    vel = k.evaluateDeviceState()
    t0, t1 = (int(t) for t in d["targets"])
    err = normalized_error(vel.x[t0:t1], vel.y[t0:t1], d["u"], d["v"])
    assert err.max() <= 1e-12


def test_symmetric_with_sub_blocks_against_ordered_and_oracle(port):
    """N = 24000 uses blocks of two 32-vortex sub-blocks (the partial rows would exceed their
    budget with one)."""
    n = 24000
    x, y, g = ics.periodic_box(n, 9, L)
    k = kernel_with(x, y, g)
    plan = k.statePlan()
    assert plan["symmetric"] and plan["rows"] == (n + 63) // 64
    vel = k.evaluateDeviceState()
    ordered = k.evaluate(x, y, g)            # host arrays: the ordered-pair kernel
    assert normalized_error(vel.x, vel.y, ordered.x, ordered.y).max() <= 1e-12
    geo = Geometry("periodic", box_length_x=L, box_length_y=L)
    u, v = port.evaluate_range(geo, x, y, g, n - 40, n)   # the ragged last block
    assert normalized_error(vel.x[n - 40:], vel.y[n - 40:], u, v).max() <= 1e-12


@pytest.mark.parametrize("n", [3000, 4100, 8192])
def test_symmetric_one_sub_block_against_ordered_and_oracle(port, n):
    """One sub-block per block (ragged last block at 3000 and 4100): every target against the
    ordered-pair kernel, three ranges against the oracle, and a repeated evaluation bit for
    bit."""
    from pointvortex_b200 import autotune
    x, y, g = ics.periodic_box(n, 31 + n, L)
    bucket = n.bit_length() - 1
    saved = autotune.get_symmetric_entry(1, 0, bucket)
    try:  # one target per lane, whatever the measured table prefers at this size
        autotune.set_symmetric_entry(1, 0, bucket, 2, 0, 0)
        k = kernel_with(x, y, g)
    finally:
        autotune.set_symmetric_entry(1, 0, bucket, *saved)
    plan = k.statePlan()
    assert plan["symmetric"] and plan["rows"] == (n + 31) // 32
    vel = k.evaluateDeviceState()
    ordered = k.evaluate(x, y, g)
    assert normalized_error(vel.x, vel.y, ordered.x, ordered.y).max() <= 1e-12
    geo = Geometry("periodic", box_length_x=L, box_length_y=L)
    for t0, t1 in ((0, 48), (n // 2 - 24, n // 2 + 24), (n - 48, n)):
        u, v = port.evaluate_range(geo, x, y, g, t0, t1)
        assert normalized_error(vel.x[t0:t1], vel.y[t0:t1], u, v).max() <= 1e-12
    again = k.evaluateDeviceState()
    assert np.array_equal(vel.x, again.x) and np.array_equal(vel.y, again.y)


def test_symmetric_coincident_pair_across_blocks_is_the_reference_error(port):
    x, y, g = ics.periodic_box(4096, 8, L)
    x[100], y[100] = x[3900], y[3900]
    k = kernel_with(x, y, g)
    xs, ys, gs = ics.periodic_box(64, 8, L)
    xs[3], ys[3] = xs[40], ys[40]
    geo = Geometry("periodic", box_length_x=L, box_length_y=L)
    with pytest.raises(RuntimeError) as want:
        port.evaluate(geo, xs, ys, gs)
    with pytest.raises(RuntimeError) as got:
        k.evaluateDeviceState()
    assert str(got.value) == str(want.value)


def test_symmetric_is_deterministic():
    x, y, g = ics.periodic_box(5000, 3, L)
    k = kernel_with(x, y, g)
    a = k.evaluateDeviceState()
    b = k.evaluateDeviceState()
    assert np.array_equal(a.x, b.x) and np.array_equal(a.y, b.y)


def test_symmetric_coincident_pair_is_the_reference_error(port):
    x, y, g = ics.periodic_box(2048, 5, L)
    x[7], y[7] = x[1500], y[1500]
    k = kernel_with(x, y, g)
    geo = Geometry("periodic", box_length_x=L, box_length_y=L)
    with pytest.raises(RuntimeError) as want:
        port.evaluate(geo, x, y, g)
    with pytest.raises(RuntimeError) as got:
        k.evaluateDeviceState()
    assert str(got.value) == str(want.value)


def test_small_populations_use_the_ordered_kernel():
    x, y, g = ics.periodic_box(1024, 2, L)
    assert not kernel_with(x, y, g).statePlan()["symmetric"]


# ---- the infinite plane (FP64 from N = 16384 up: four targets per lane off the diagonal, eight
# from N = 32768 up) -----------------------------------------------------------------------------

def plane_kernel_with(x, y, g, core=0.0):
    k = pv.InfinitePlaneKernel(core)
    k.uploadDeviceState(pv.VortexSystem(x, y, g))
    return k


@pytest.mark.parametrize("n,core", [(16384, 0.0), (16400, 0.0), (20000, 0.05)])
def test_plane_symmetric_matches_oracle(reference, n, core):
    """16400 and 20000 end in a ragged block (blocks of 32 vortices per target of a lane, 128 or
    256 as the tables choose); 0.05 is a core radius."""
    x, y, g = ics.infinite_plane(n, 70 + n)
    k = plane_kernel_with(x, y, g, core)
    plan = k.statePlan()
    block = 32 * plan["symmetric_targets"]  # 4 or 8 targets per lane, as the tables choose
    assert plan["symmetric"] and plan["rows"] == (n + block - 1) // block
    vel = k.evaluateDeviceState()
    u, v = reference.evaluate(Geometry("infinite", core_radius=core), x, y, g)
    assert normalized_error(vel.x, vel.y, u, v).max() <= 1e-12


@pytest.mark.parametrize("n", [33000, 40000])
def test_plane_symmetric_wide_against_ordered_and_oracle(port, n):
    """Eight targets per lane (256-vortex blocks, ragged last block): all targets against the
    ordered-pair kernel, the first and the last ones against the oracle."""
    x, y, g = ics.infinite_plane(n, 17)
    k = plane_kernel_with(x, y, g)
    plan = k.statePlan()
    block = 32 * plan["symmetric_targets"]
    assert plan["symmetric"] and plan["rows"] == (n + block - 1) // block
    vel = k.evaluateDeviceState()
    ordered = k.evaluate(x, y, g)
    assert normalized_error(vel.x, vel.y, ordered.x, ordered.y).max() <= 1e-12
    geo = Geometry("infinite")
    for t0, t1 in ((0, 40), (n - 40, n)):
        u, v = port.evaluate_range(geo, x, y, g, t0, t1)
        assert normalized_error(vel.x[t0:t1], vel.y[t0:t1], u, v).max() <= 1e-12


def test_plane_symmetric_is_deterministic():
    x, y, g = ics.infinite_plane(17000, 4)
    k = plane_kernel_with(x, y, g)
    a = k.evaluateDeviceState()
    b = k.evaluateDeviceState()
    assert np.array_equal(a.x, b.x) and np.array_equal(a.y, b.y)


@pytest.mark.parametrize("n,i,j", [(16384, 7, 16000), (16384, 130, 131), (33000, 9, 32990)])
def test_plane_symmetric_coincident_pair_is_the_reference_error(port, n, i, j):
    """Off the diagonal and inside one sub-block; the oracle's error comes from a 64-vortex system
    with the same coincidence."""
    x, y, g = ics.infinite_plane(n, 5)
    x[i], y[i] = x[j], y[j]
    k = plane_kernel_with(x, y, g)
    xs, ys, gs = ics.infinite_plane(64, 5)
    xs[3], ys[3] = xs[40], ys[40]
    with pytest.raises(RuntimeError) as want:
        port.evaluate(Geometry("infinite"), xs, ys, gs)
    with pytest.raises(RuntimeError) as got:
        k.evaluateDeviceState()
    assert str(got.value) == str(want.value)


def test_plane_coincident_pair_with_core_is_finite(reference):
    x, y, g = ics.infinite_plane(16384, 6)
    x[9], y[9] = x[5000], y[5000]
    k = plane_kernel_with(x, y, g, 0.01)
    vel = k.evaluateDeviceState()
    u, v = reference.evaluate(Geometry("infinite", core_radius=0.01), x, y, g)
    assert normalized_error(vel.x, vel.y, u, v).max() <= 1e-12


def test_small_plane_populations_use_the_ordered_kernel():
    x, y, g = ics.infinite_plane(16000, 2)
    assert not plane_kernel_with(x, y, g).statePlan()["symmetric"]


@pytest.mark.parametrize("n", [17000, 33000])
def test_plane_fp32c_symmetric_against_the_fp64_oracle(port, n):
    """The FP32-compensated plane once per unordered pair (4 targets per lane at 17000, 8 at
    33000) against the FP64 ordered kernel: no worse than the ordered FP32C kernel on the same
    state (max within 2x, rms within 1.5x, or the FP32C bounds 2e-6 / 2e-7 of smaller
    populations), and at most 1e-5 anywhere; three ranges against the oracle."""
    x, y, g = ics.infinite_plane(n, 23)
    k = pv.InfinitePlaneKernel(0.0, precision=_lib.PRECISION_FP32C)
    k.uploadDeviceState(pv.VortexSystem(x, y, g))
    plan = k.statePlan()
    block = 32 * plan["symmetric_targets"]
    assert plan["symmetric"] and plan["rows"] == (n + block - 1) // block
    vel = k.evaluateDeviceState()
    ref = pv.InfinitePlaneKernel(0.0).evaluate(x, y, g)
    err = normalized_error(vel.x, vel.y, ref.x, ref.y)
    ordered = k.evaluate(x, y, g)            # host arrays: the ordered FP32C kernel
    err_o = normalized_error(ordered.x, ordered.y, ref.x, ref.y)
    rms, rms_o = np.sqrt(np.mean(err ** 2)), np.sqrt(np.mean(err_o ** 2))
    assert err.max() <= min(max(2.0 * err_o.max(), 2e-6), 1e-5)
    assert rms <= min(max(1.5 * rms_o, 2e-7), 1e-6)
    geo = Geometry("infinite")
    for t0, t1 in ((0, 40), (n // 2, n // 2 + 40), (n - 40, n)):
        u, v = port.evaluate_range(geo, x, y, g, t0, t1)
        assert normalized_error(vel.x[t0:t1], vel.y[t0:t1], u, v).max() <= 1e-5
    again = k.evaluateDeviceState()
    assert np.array_equal(vel.x, again.x) and np.array_equal(vel.y, again.y)


def test_small_plane_fp32c_uses_the_ordered_kernel():
    x, y, g = ics.infinite_plane(16000, 2)
    k = pv.InfinitePlaneKernel(0.0, precision=_lib.PRECISION_FP32C)
    k.uploadDeviceState(pv.VortexSystem(x, y, g))
    assert not k.statePlan()["symmetric"]


def test_tuning_table_changes_the_plan_and_keeps_parity(port):
    """An entry of the symmetric-form table changes the plan the context chooses (pv_state_plan):
    the ordered kernel instead of the symmetric form, or the periodic kernel built for 7 or 8 CTAs
    per SM; every choice stays within the parity tolerance of the oracle."""
    from pointvortex_b200 import autotune
    x, y, g = ics.periodic_box(4096, 91, 2.0)
    geo = Geometry("periodic", box_length_x=2.0, box_length_y=2.0)
    ur, vr = port.evaluate(geo, x, y, g)
    seen = []
    saved = autotune.get_symmetric_entry(1, 0, 12)
    try:
        for entry in [(1,), (2, 7), (2, 8), (2, 0, 2), (0,)]:
            autotune.set_symmetric_entry(1, 0, 12, *entry)
            k = pv.PeriodicBoxKernel(2.0, 2.0, 8)
            k.uploadDeviceState(pv.VortexSystem(x, y, g))
            plan = k.statePlan()
            seen.append((plan["symmetric"], plan["symmetric_min_ctas"],
                         plan["symmetric_targets"] if plan["symmetric"] else 0))
            f = k.evaluateDeviceState()
            assert normalized_error(f.x, f.y, ur, vr).max() <= 1e-12, entry
            k.close()
    finally:
        autotune.set_symmetric_entry(1, 0, 12, *saved)
    assert seen == [(False, 0, 0), (True, 7, 1), (True, 8, 1), (True, 0, 2), (True, 0, 1)]


def test_grid_table_changes_the_grid_and_keeps_the_result(port):
    """An entry of the grid table (pv_set_symmetric_grid) changes the persistent grid's CTAs per
    SM (pv_state_plan), clamped to what fits; the velocities are bit for bit the same, since
    every (row, vortex) entry is written by one item whichever warp takes it."""
    from pointvortex_b200 import autotune
    x, y, g = ics.periodic_box(4096, 93, 2.0)
    saved = autotune.get_symmetric_entry(1, 0, 12), autotune.get_symmetric_grid(1, 0, 12)
    out = []
    try:
        autotune.set_symmetric_entry(1, 0, 12, 2)
        for ctas in (0, 3, 16):
            autotune.set_symmetric_grid(1, 0, 12, ctas)
            k = pv.PeriodicBoxKernel(2.0, 2.0, 8)
            k.uploadDeviceState(pv.VortexSystem(x, y, g))
            out.append((k.statePlan()["symmetric_grid_ctas"], k.evaluateDeviceState()))
            k.close()
    finally:
        autotune.set_symmetric_entry(1, 0, 12, *saved[0])
        autotune.set_symmetric_grid(1, 0, 12, saved[1])
    fit = out[0][0]
    assert fit >= 4 and out[1][0] == 3 and out[2][0] == fit
    for _, f in out[1:]:
        assert np.array_equal(f.x, out[0][1].x) and np.array_equal(f.y, out[0][1].y)
    geo = Geometry("periodic", box_length_x=2.0, box_length_y=2.0)
    u, v = port.evaluate_range(geo, x, y, g, 0, 64)
    assert normalized_error(out[1][1].x[:64], out[1][1].y[:64], u, v).max() <= 1e-12


def test_periodic_two_targets_per_lane_ragged_against_ordered_and_oracle(port):
    """The periodic kernel with two targets per lane (blocks of 64, table entry targets = 2) on a
    population that ends inside a block: the same velocities as the oracle and the ordered
    kernel, within the parity tolerance."""
    from pointvortex_b200 import autotune
    n = 4136
    x, y, g = ics.periodic_box(n, 92, 2.0)
    geo = Geometry("periodic", box_length_x=2.0, box_length_y=2.0)
    saved = autotune.get_symmetric_entry(1, 0, 12)
    try:
        autotune.set_symmetric_entry(1, 0, 12, 2, 0, 2)
        k = pv.PeriodicBoxKernel(2.0, 2.0, 8)
        k.uploadDeviceState(pv.VortexSystem(x, y, g))
        plan = k.statePlan()
        assert plan["symmetric"] and plan["symmetric_targets"] == 2
        f = k.evaluateDeviceState()
        ordered = k.evaluate(x, y, g)
        k.close()
    finally:
        autotune.set_symmetric_entry(1, 0, 12, *saved)
    assert normalized_error(f.x, f.y, ordered.x, ordered.y).max() <= 1e-12
    for t0, t1 in ((0, 64), (n - 72, n)):
        u, v = port.evaluate_range(geo, x, y, g, t0, t1)
        assert normalized_error(f.x[t0:t1], f.y[t0:t1], u, v).max() <= 1e-12
