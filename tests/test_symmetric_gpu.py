"""The periodic box evaluated once per unordered pair (the device-state path from N = 2048 up):
against the oracle and against the ordered-pair kernel, on ragged populations, with more than one
sub-block per block (N = 24000), deterministic, and with the reference's errors."""
import numpy as np
import pytest

import pointvortex_b200 as pv
from conftest import golden, normalized_error
from oracle.pyoracle import Geometry
from pointvortex_b200 import ics

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
