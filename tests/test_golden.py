"""The oracle (C restatement) against the reference's known-answer tests and against the golden
fixtures generated from the unmodified reference (tests/golden/make_golden.py). CPU only."""
import numpy as np
import pytest

import known_answers
from conftest import golden
from oracle.pyoracle import Geometry


class PortImpl:
    def __init__(self, port):
        self.o = port

    def evaluate(self, geo, x, y, g):
        return self.o.evaluate(geo, x, y, g)

    def hamiltonian(self, geo, x, y, g):
        return self.o.hamiltonian(geo, x, y, g)

    def stepper(self, geo, n):
        return self.o.stepper(geo, n)


@pytest.mark.parametrize("case", known_answers.ALL, ids=lambda f: f.__name__)
def test_known_answers_on_oracle(port, case):
    case(PortImpl(port))


SMALL = {
    "infinite": Geometry("infinite"),
    "infinite_core": Geometry("infinite", core_radius=0.05),
    "periodic": Geometry("periodic", box_length_x=2.0, box_length_y=2.0),
    "periodic_m3": Geometry("periodic", box_length_x=2.0, box_length_y=2.0, image_layers=3),
    "disk": Geometry("disk", disk_radius=1.0),
}


@pytest.mark.parametrize("tag", sorted(SMALL))
def test_small_fixtures_bit_exact(port, tag):
    d = golden(f"small_{tag}.npz")
    geo = SMALL[tag]
    x, y, g = d["x"], d["y"], d["g"]
    u, v = port.evaluate(geo, x, y, g)
    assert np.array_equal(u, d["u"]) and np.array_equal(v, d["v"])
    assert np.array_equal(port.invariants(geo, x, y, g), d["inv"])
    st = port.stepper(geo, x.size)
    for k in range(3):
        nx, ny = st.rk4_step(d["rk_x"][k], d["rk_y"][k], g, 1e-3)
        assert np.array_equal(nx, d["rk_x"][k + 1]) and np.array_equal(ny, d["rk_y"][k + 1])
    dp = port.stepper(geo, x.size)
    cx, cy, dt = x, y, 1e-3
    for k in range(3):
        cx, cy, r = dp.dopri5_step(cx, cy, g, dt)
        assert np.array_equal(cx, d["dp_x"][k + 1]) and np.array_equal(r, d["dp_r"][k])
        dt = r[1]


def test_workload_fixtures(port):
    d = golden("workload_infinite_n1024.npz")
    geo = Geometry("infinite")
    u, v = port.evaluate(geo, d["x"], d["y"], d["g"])
    assert np.array_equal(u, d["u"]) and np.array_equal(v, d["v"])
    st = port.stepper(geo, d["x"].size)
    nx, ny = st.rk4_step(d["rk_x"][2], d["rk_y"][2], d["g"], 1e-3)
    assert np.array_equal(nx, d["rk_x"][3]) and np.array_equal(ny, d["rk_y"][3])
    d = golden("workload_periodic_n4096.npz")
    geo = Geometry("periodic", box_length_x=2 * np.pi, box_length_y=2 * np.pi)
    u, v = port.evaluate_range(geo, d["x"], d["y"], d["g"], 0, 64)
    assert np.array_equal(u, d["u"][:64]) and np.array_equal(v, d["v"][:64])
    d = golden("workload_disk_n16384.npz")
    geo = Geometry("disk", disk_radius=1.0)
    u, v = port.evaluate_range(geo, d["x"], d["y"], d["g"], 0, 256)
    assert np.array_equal(u, d["u"]) and np.array_equal(v, d["v"])
