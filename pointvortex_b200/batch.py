"""Batched ensembles over libpvb200's pv_batch_* API.

Many independent simulations (each: geometry, population, precision form, tolerances, end time)
share one device arena and advance in lock-step DOPRI5 attempts, each with its own step size. A
simulation's result is the same alone and in any mix.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import lib
from .kernel import CudaError, _EXCEPTIONS, _f64, _ptr

STATES = {_lib.SIM_RUNNING: "running", _lib.SIM_DONE: "done", _lib.SIM_FAILED: "failed",
          _lib.SIM_BUDGET: "budget"}


class CapacityError(RuntimeError):
    """Admission refused: no free slot or no room in the batch arena."""


# Why a failed simulation stopped: the device status code (and, for the integrator's failure, which
# of its conditions), named after the reference's checks.
_STATUS_REASONS = {2: "outside_disk", 3: "nonfinite_position", 4: "nonfinite_error_estimate",
                   5: "nonfinite_velocity", 6: "coincident", 10: "timeout"}
_INTEGRATOR_FAILURES = {1: "rejection_cap", 2: "dt_floor", 3: "no_time_advance"}


@dataclass
class SimInfo:
    state: str
    status: int
    time: float
    suggestedTimeStep: float
    acceptedSteps: int
    rejectedSteps: int
    population: int
    failure: int = 0
    targetsPerThread: int = 0  # of the ordered work items; 0: once-per-unordered-pair items

    @property
    def reason(self) -> str:
        """"done", "budget", "running", or the failure: rejection_cap (more than 32 rejections
        in one step), dt_floor (rejected at the minimum step), no_time_advance (src/timestep.cpp:
        116-117, src/main.cpp:314-315), outside_disk (src/compute.cpp:41-48), coincident,
        nonfinite_velocity, nonfinite_position, nonfinite_error_estimate, timeout."""
        if self.state != "failed":
            return self.state
        if self.status == 1:
            return _INTEGRATOR_FAILURES.get(self.failure, "integrator")
        return _STATUS_REASONS.get(self.status, f"status_{self.status}")


PRECISIONS = {"fp64": _lib.PRECISION_FP64, "fp32c": _lib.PRECISION_FP32C}


def geometry_params(boundary: str, core_radius: float = 0.0, box_length: float = 2.0 * np.pi,
                    image_layers: int = 8, disk_radius: float = 1.0,
                    precision: str = "fp64") -> _lib.PvParams:
    """Parameters of one batched simulation; precision "fp64" (plain) or "fp32c" (the
    FP32-compensated form)."""
    g = {"infinite": _lib.GEOMETRY_INFINITE, "periodic": _lib.GEOMETRY_PERIODIC,
         "disk": _lib.GEOMETRY_DISK}[boundary]
    return _lib.PvParams(g, core_radius, box_length, box_length, image_layers, disk_radius,
                         PRECISIONS[precision])


class Batch:
    def __init__(self, capacity_vortices: int, max_simulations: int, device: int = 0,
                 max_steps: int = 0, partial_factor: int = 0):
        cfg = _lib.PvBatchConfig(capacity_vortices, max_simulations, device, max_steps,
                                 partial_factor)
        self._b = ctypes.c_void_p()
        rc = lib.pv_batch_create(ctypes.byref(cfg), ctypes.byref(self._b))
        if rc != _lib.PV_OK:
            raise _EXCEPTIONS.get(rc, RuntimeError)(lib.pv_last_error(None).decode())

    def close(self):
        if getattr(self, "_b", None) and self._b.value:
            lib.pv_batch_destroy(self._b)
            self._b = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc == _lib.PV_ERROR_CAPACITY:
            raise CapacityError(lib.pv_batch_last_error(self._b).decode())
        if rc != _lib.PV_OK:
            raise _EXCEPTIONS.get(rc, RuntimeError)(lib.pv_batch_last_error(self._b).decode())

    def add(self, params: _lib.PvParams, x, y, circulation, t_end: float, dt: float = 1e-3,
            atol: float = 1e-10, rtol: float = 1e-8, dtmin: float = 1e-12, dtmax: float = 0.1,
            max_steps: int = 0) -> int:
        x, y, g = _f64(x), _f64(y), _f64(circulation)
        solve = _lib.PvBatchSolve(t_end, dt, atol, rtol, dtmin, dtmax, max_steps)
        sid = ctypes.c_uint32(0)
        self._check(lib.pv_batch_add(self._b, ctypes.byref(params), _ptr(x), _ptr(y), _ptr(g),
                                     x.size, ctypes.byref(solve), ctypes.byref(sid)))
        return int(sid.value)

    def advance(self, attempts: int = 1) -> int:
        running = ctypes.c_uint32(0)
        self._check(lib.pv_batch_advance(self._b, attempts, ctypes.byref(running)))
        return int(running.value)

    def run(self, max_attempts: int = 1 << 30, chunk: int = 8) -> int:
        """Advances until no simulation is running (or max_attempts); returns attempts made."""
        made = 0
        while made < max_attempts:
            k = min(chunk, max_attempts - made)
            running = self.advance(k)
            made += k
            if running == 0:
                break
        return made

    def info(self, sid: int) -> SimInfo:
        i = _lib.PvBatchSimInfo()
        self._check(lib.pv_batch_info(self._b, sid, ctypes.byref(i)))
        return SimInfo(STATES.get(i.state, "free"), i.status, i.time, i.suggested_time_step,
                       int(i.accepted_steps), int(i.rejected_steps), int(i.population),
                       int(i.failure), int(i.targets_per_thread))

    def result(self, sid: int):
        n = self.info(sid).population
        x = np.empty(n)
        y = np.empty(n)
        self._check(lib.pv_batch_result(self._b, sid, _ptr(x), _ptr(y), n))
        return x, y

    def release(self, sid: int) -> None:
        self._check(lib.pv_batch_release(self._b, sid))

    def totals(self) -> dict:
        t = _lib.PvBatchTotals()
        self._check(lib.pv_batch_status(self._b, ctypes.byref(t)))
        return {"attempts": int(t.attempts), "work_items": int(t.work_items),
                "free_vortices": int(t.free_vortices), "running": int(t.running),
                "occupied_slots": int(t.occupied_slots)}

    def cudaStream(self) -> int:
        s = ctypes.c_void_p()
        self._check(lib.pv_batch_stream(self._b, ctypes.byref(s)))
        return int(s.value or 0)
