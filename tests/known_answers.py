"""The reference's own known-answer tests (tests/tests.cpp and tests/audit_tests.cpp of
jplaurie/PointVortex), written once against a small adapter so that they run on the oracle
(test_golden.py, CPU) and on the CUDA path (test_known_answers_gpu.py, B200).

An implementation adapter provides
    evaluate(geo, x, y, g) -> (u, v)                 VelocityKernel::evaluate
    hamiltonian(geo, x, y, g) -> float               VelocityKernel::hamiltonian
    stepper(geo, n) -> object with rk4_step(x, y, g, dt) -> (x, y),
                       dopri5_step(x, y, g, dt) -> (x, y, [dt, suggested, error, rejected]),
                       invalidate(), evaluations    RungeKuttaIntegrator
and raises ValueError / IndexError / RuntimeError like the reference's exception types.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from oracle.pyoracle import Geometry

INV2PI = 0.5 / math.pi


def near(got, want, tol, what):
    assert math.isfinite(got) and math.isfinite(want) and abs(got - want) <= tol, (what, got, want)


def pair():
    return np.array([-1.0, 1.0]), np.array([0.0, 0.0]), np.array([1.0, 1.0])


def velocity_tests(impl):
    """tests/tests.cpp:26-41"""
    plane = Geometry("infinite")
    u, v = impl.evaluate(plane, [2.0], [-3.0], [4.0])
    assert u[0] == 0.0 and v[0] == 0.0
    u, v = impl.evaluate(plane, *pair())
    speed = 1.0 / (4.0 * math.pi)
    near(v[0], -speed, 1e-15, "pair v0")
    near(v[1], speed, 1e-15, "pair v1")


def rk4_test(impl):
    """tests/tests.cpp:42-51"""
    x, y, g = pair()
    st = impl.stepper(Geometry("infinite"), 2)
    for _ in range(1000):
        x, y = st.rk4_step(x, y, g, 1e-3)
    angle = 1.0 / (4.0 * math.pi)
    near(x[1], math.cos(angle), 2e-12, "RK4 x")
    near(y[1], math.sin(angle), 2e-12, "RK4 y")


def dopri_test(impl):
    """tests/tests.cpp:52-70"""
    x, y, g = pair()
    geo = Geometry("infinite", absolute_tolerance=1e-12, relative_tolerance=1e-10,
                   minimum_time_step=1e-12, maximum_time_step=0.2)
    st = impl.stepper(geo, 2)
    time, dt = 0.0, 0.01
    while time < 1.0:
        x, y, r = st.dopri5_step(x, y, g, min(dt, 1.0 - time))
        time += r[0]
        dt = r[1]
    angle = 1.0 / (4.0 * math.pi)
    near(x[1], math.cos(angle), 2e-10, "DOPRI x")
    near(y[1], math.sin(angle), 2e-10, "DOPRI y")


def geometry_tests(impl):
    """tests/tests.cpp:126-154"""
    box = Geometry("periodic", box_length_x=2.0, box_length_y=2.0, image_layers=10)
    x = np.array([-0.4, 0.4])
    y = np.array([0.1, -0.1])
    g = np.array([1.0, -1.0])
    u1, v1 = impl.evaluate(box, x, y, g)
    x2, y2 = x.copy(), y.copy()
    x2[0] += 2.0
    y2[1] -= 2.0
    u2, v2 = impl.evaluate(box, x2, y2, g)
    for i in range(2):
        near(u2[i], u1[i], 2e-14, "periodic u invariance")
        near(v2[i], v1[i], 2e-14, "periodic v invariance")
    circle = Geometry("disk", disk_radius=2.0)
    u, v = impl.evaluate(circle, [0.5], [0.0], [1.0])
    near(u[0], 0.0, 1e-15, "disk radial velocity")
    near(v[0], 0.5 / (2.0 * math.pi * (4.0 - 0.25)), 1e-15, "disk image velocity")
    energy = impl.hamiltonian(circle, [0.5], [0.0], [1.0])
    st = impl.stepper(circle, 1)
    dx, dy = np.array([0.5]), np.array([0.0])
    for _ in range(100):
        dx, dy = st.rk4_step(dx, dy, np.array([1.0]), 1e-3)
    near(impl.hamiltonian(circle, dx, dy, [1.0]), energy, 2e-15, "disk Hamiltonian")


def fsal_test(impl):
    """tests/tests.cpp:297-314 (the CountingKernel counts evaluations: 7, 13, 20)."""
    x, y, g = pair()
    geo = Geometry("infinite", absolute_tolerance=1e-10, relative_tolerance=1e-8)
    st = impl.stepper(geo, 2)
    x, y, _ = st.dopri5_step(x, y, g, 1e-3)
    assert st.evaluations == 7
    x, y, _ = st.dopri5_step(x, y, g, 1e-3)
    assert st.evaluations == 13
    st.invalidate()
    st.dopri5_step(x, y, g, 1e-3)
    assert st.evaluations == 20


def close_encounter_tests(impl):
    """tests/audit_tests.cpp:27-49"""
    box = Geometry("periodic", box_length_x=2.0, box_length_y=2.0)
    x = np.array([0.0, 1e-10])
    y = np.array([0.0, 0.0])
    g = np.array([1.0, -1.0])
    u, v = impl.evaluate(box, x, y, g)
    near(v[0] / (INV2PI / 1e-10), 1.0, 1e-12, "close periodic pair")
    assert math.isfinite(impl.hamiltonian(box, x, y, g))
    with pytest.raises(RuntimeError):
        impl.evaluate(box, np.array([0.0, 0.0]), y, g)
    disk = Geometry("disk", disk_radius=1.0)
    x = np.array([0.2, 1e-155])
    u, v = impl.evaluate(disk, x, y, np.array([1.0, 1.0]))
    near(u[0], 0.0, 1e-15, "near-center disk radial velocity")
    near(v[0], INV2PI * (5 + 0.2 / 0.96), 1e-14, "near-center disk tangential velocity")
    near(v[1], INV2PI * (-5 + 0.2), 1e-14, "near-center source image")
    with pytest.raises(ValueError):
        impl.evaluate(Geometry("periodic", box_length_x=2.0, box_length_y=2.0, image_layers=65),
                      x, y, g)


def hamiltonian_tests(impl):
    """tests/audit_tests.cpp:51-85: velocity = Hamiltonian gradient; H conservation."""
    x = np.array([-0.31, 0.23, 0.11, -0.14])
    y = np.array([-0.12, 0.14, -0.29, 0.32])
    g = np.array([1.0, -1.0, 2.0, -2.0])
    for geo in (Geometry("infinite", core_radius=0.05),
                Geometry("periodic", box_length_x=2.0, box_length_y=2.0),
                Geometry("disk", disk_radius=1.0)):
        u, v = impl.evaluate(geo, x, y, g)
        h = 1e-6
        for i in range(4):
            xp, xm = x.copy(), x.copy()
            xp[i] += h
            xm[i] -= h
            dx = (impl.hamiltonian(geo, xp, y, g) - impl.hamiltonian(geo, xm, y, g)) / (2 * h)
            yp, ym = y.copy(), y.copy()
            yp[i] += h
            ym[i] -= h
            dy = (impl.hamiltonian(geo, x, yp, g) - impl.hamiltonian(geo, x, ym, g)) / (2 * h)
            near(u[i], dy / g[i], 2e-8, "Hamiltonian u derivative")
            near(v[i], -dx / g[i], 2e-8, "Hamiltonian v derivative")
        st = impl.stepper(geo, 4)
        ex, ey = x.copy(), y.copy()
        for _ in range(100):
            ex, ey = st.rk4_step(ex, ey, g, 1e-4)
        near(impl.hamiltonian(geo, ex, ey, g), impl.hamiltonian(geo, x, y, g), 1e-10,
             "multi-vortex Hamiltonian conservation")


def invalid_numeric_tests(impl):
    """tests/audit_tests.cpp:99-118 (the parts that reach the velocity path)."""
    plane = Geometry("infinite")
    st = impl.stepper(plane, 1)
    with pytest.raises(ValueError):
        st.rk4_step(np.array([0.0]), np.array([0.0]), np.array([1.0]), 0.0)
    with pytest.raises(ValueError):
        impl.evaluate(plane, [math.nan], [0.0], [1.0])


ALL = [velocity_tests, rk4_test, dopri_test, geometry_tests, fsal_test, close_encounter_tests,
       hamiltonian_tests, invalid_numeric_tests]
