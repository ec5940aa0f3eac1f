"""Seeded synthetic initial conditions with the shapes and distributions of the benchmark
workloads (the reference has no dataset; these stand in for its parameter-file cases).

    infinite plane : x, y ~ U[-1, 1]^2, Gamma = +-1 with exactly N/2 of each sign, shuffled
    periodic box   : x, y ~ U[-L/2, L/2)^2 (the reference's box convention, src/read.cpp:291-305),
                     Gamma = +-1 balanced (zero net circulation)
    disk           : r = a R sqrt(U), theta = 2 pi U (uniform by area in r <= a R),
                     Gamma ~ N(0, 1) or +-1 balanced

Every generator returns (x, y, circulation) as float64 numpy arrays.
"""
from __future__ import annotations

import numpy as np


def balanced_signs(n: int, rng: np.random.Generator) -> np.ndarray:
    g = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
    rng.shuffle(g)
    return g


def infinite_plane(n: int, seed: int, half_width: float = 1.0):
    rng = np.random.default_rng(seed)
    x = rng.uniform(-half_width, half_width, n)
    y = rng.uniform(-half_width, half_width, n)
    return x, y, balanced_signs(n, rng)


def periodic_box(n: int, seed: int, length: float = 2.0 * np.pi):
    if n % 2:
        raise ValueError("a balanced periodic population needs an even N")
    rng = np.random.default_rng(seed)
    x = rng.uniform(-0.5 * length, 0.5 * length, n)
    y = rng.uniform(-0.5 * length, 0.5 * length, n)
    return x, y, balanced_signs(n, rng)


def disk(n: int, seed: int, radius: float = 1.0, fill: float = 0.95, gaussian: bool = True):
    rng = np.random.default_rng(seed)
    r = fill * radius * np.sqrt(rng.random(n))
    th = 2.0 * np.pi * rng.random(n)
    g = rng.standard_normal(n) if gaussian else balanced_signs(n, rng)
    return r * np.cos(th), r * np.sin(th), g


# The three single-simulation workloads (sizes, geometry parameters, integrator settings).
WORKLOADS = {
    "infinite_rk4_n1024": dict(geometry="infinite", n=1024, seed=20240101, integrator="rk4",
                               dt=1e-3, steps=100),
    "periodic_dopri5_n4096": dict(geometry="periodic", n=4096, seed=20240102, length=2 * np.pi,
                                  integrator="dopri5", dt=1e-3, rtol=1e-9, atol=1e-12,
                                  t_end=1.0, dipole_threshold=1e-3),
    "disk_rk4_n16384": dict(geometry="disk", n=16384, seed=20240103, radius=1.0,
                            integrator="rk4", dt=5e-4, steps=200),
}


def workload_state(name: str):
    """(x, y, circulation) of a named workload."""
    w = WORKLOADS[name]
    if w["geometry"] == "infinite":
        return infinite_plane(w["n"], w["seed"])
    if w["geometry"] == "periodic":
        return periodic_box(w["n"], w["seed"], w["length"])
    return disk(w["n"], w["seed"], w["radius"])
