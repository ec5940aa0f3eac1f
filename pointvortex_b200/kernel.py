"""Host-side mirror of the reference's velocity-backend interface, over libpvb200.

Names, argument meaning and error behaviour follow jplaurie/PointVortex:

* ``VortexSystem`` / ``VelocityField``          -- src/vortex.h:15-51 (structure of arrays)
* ``VelocityKernel`` and its three geometries    -- src/compute.h:18-75
* ``StepResult``                                 -- src/compute.h:11-16
* ``Invariants`` / ``computeInvariants``         -- src/compute.h:76-84
* ``makeBackendKernel`` / ``backendName`` /
  ``backendRuntimeDetails``                      -- src/backend.h:9-16

Exceptions map the reference's C++ types: std::invalid_argument -> ValueError,
std::out_of_range -> IndexError, std::runtime_error -> RuntimeError, std::logic_error ->
LogicError (a RuntimeError subclass). All arithmetic runs on the GPU; constructing a kernel on a
machine without a CUDA device raises CudaError.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import _lib
from ._lib import lib


class LogicError(RuntimeError):
    """std::logic_error: a device-stepping hook used before the state was uploaded."""


class CudaError(RuntimeError):
    """A CUDA runtime call failed (no device, out of memory, ...)."""


_EXCEPTIONS = {
    _lib.PV_ERROR_INVALID_ARGUMENT: ValueError,
    _lib.PV_ERROR_OUT_OF_RANGE: IndexError,
    _lib.PV_ERROR_RUNTIME: RuntimeError,
    _lib.PV_ERROR_LOGIC: LogicError,
    _lib.PV_ERROR_CUDA: CudaError,
}

_DP = ctypes.POINTER(ctypes.c_double)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_DP)


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


@dataclass
class VortexSystem:
    """Structure-of-arrays vortex state (src/vortex.h:15-38)."""

    x: np.ndarray = field(default_factory=lambda: np.zeros(0))
    y: np.ndarray = field(default_factory=lambda: np.zeros(0))
    circulation: np.ndarray = field(default_factory=lambda: np.zeros(0))

    def __post_init__(self):
        self.x, self.y, self.circulation = _f64(self.x), _f64(self.y), _f64(self.circulation)

    def size(self) -> int:
        return int(self.x.size)

    def copy(self) -> "VortexSystem":
        return VortexSystem(self.x.copy(), self.y.copy(), self.circulation.copy())

    def validate(self) -> None:
        """validateVortexArrays (src/vortex.h:7-14)."""
        if not (self.x.size == self.y.size == self.circulation.size):
            raise ValueError("vortex arrays have different lengths")
        if not (np.isfinite(self.x).all() and np.isfinite(self.y).all()
                and np.isfinite(self.circulation).all()):
            raise ValueError("vortex data must be finite")


@dataclass
class VelocityField:
    """(u, v) per vortex (src/vortex.h:39-51)."""

    x: np.ndarray = field(default_factory=lambda: np.zeros(0))
    y: np.ndarray = field(default_factory=lambda: np.zeros(0))

    def size(self) -> int:
        return int(self.x.size)


@dataclass
class StepResult:
    """src/compute.h:11-16."""

    acceptedTimeStep: float = 0.0
    suggestedTimeStep: float = 0.0
    normalizedError: float = 0.0
    rejectedSteps: int = 0


@dataclass
class Invariants:
    """src/compute.h:76-79."""

    circulation: float = 0.0
    linearImpulseX: float = 0.0
    linearImpulseY: float = 0.0
    angularImpulse: float = 0.0
    hamiltonian: float = 0.0

    @classmethod
    def from_array(cls, a) -> "Invariants":
        return cls(*(float(v) for v in a))


@dataclass
class DipoleCandidate:
    """One candidate of the close-dipole scan (src/dipole.cpp:53-57); second == population marks
    a disk wall-image candidate."""

    first: int
    second: int
    distanceSquared: float


class VelocityKernel:
    """A B200 context behind the reference's VelocityKernel interface (src/compute.h:18-36)."""

    def __init__(self, geometry: int, *, core_radius: float = 0.0, box_length_x: float = 2.0,
                 box_length_y: float = 2.0, image_layers: int = 8, disk_radius: float = 1.0,
                 precision: int = _lib.PRECISION_FP64, device: int = 0):
        self._params = _lib.PvParams(geometry, core_radius, box_length_x, box_length_y,
                                     image_layers, disk_radius, precision)
        self._ctx = ctypes.c_void_p()
        rc = lib.pv_context_create(ctypes.byref(self._params), device, ctypes.byref(self._ctx))
        if rc != _lib.PV_OK:
            msg = lib.pv_last_error(None).decode()
            raise _EXCEPTIONS.get(rc, RuntimeError)(msg)
        self.device = device

    # -- plumbing ------------------------------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_ctx", None) and self._ctx.value:
            lib.pv_context_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int) -> None:
        if rc != _lib.PV_OK:
            msg = lib.pv_last_error(self._ctx).decode()
            raise _EXCEPTIONS.get(rc, RuntimeError)(msg)

    @staticmethod
    def _arrays(*args):
        if len(args) == 1:
            s = args[0]
            x, y, g = s.x, s.y, s.circulation
        else:
            x, y, g = args
        x, y, g = _f64(x), _f64(y), _f64(g)
        if not (x.shape == y.shape == g.shape):
            raise ValueError("vortex arrays have different lengths")
        return x, y, g

    # -- VelocityKernel ------------------------------------------------------------------------
    def evaluate(self, *args) -> VelocityField:
        """evaluate(vortices) or evaluate(x, y, circulation): src/compute.cpp:57-69."""
        x, y, g = self._arrays(*args)
        n = x.size
        u = np.empty(max(n, 1))
        v = np.empty(max(n, 1))
        self._check(lib.pv_evaluate(self._ctx, _ptr(x), _ptr(y), _ptr(g), n, _ptr(u), _ptr(v)))
        return VelocityField(u[:n], v[:n])

    def evaluateRange(self, x, y, circulation, velocity: Optional[VelocityField] = None,
                      begin: int = 0, end: Optional[int] = None) -> VelocityField:
        """src/compute.h:26-28: fills velocity[begin:end) (resized to N) with the velocities of
        those targets due to all N sources."""
        x, y, g = self._arrays(x, y, circulation)
        n = x.size
        end = n if end is None else end
        if velocity is None or velocity.size() != n:
            velocity = VelocityField(np.zeros(n), np.zeros(n))
        if begin < 0 or end < 0:
            raise IndexError("invalid target-vortex range")
        k = max(end - begin, 0)
        u = np.empty(max(k, 1))
        v = np.empty(max(k, 1))
        self._check(lib.pv_evaluate_range(self._ctx, _ptr(x), _ptr(y), _ptr(g), n, begin, end,
                                          _ptr(u), _ptr(v)))
        velocity.x[begin:end] = u[:k]
        velocity.y[begin:end] = v[:k]
        return velocity

    def hamiltonian(self, vortices: VortexSystem) -> float:
        x, y, g = self._arrays(vortices)
        out = ctypes.c_double(0.0)
        self._check(lib.pv_hamiltonian(self._ctx, _ptr(x), _ptr(y), _ptr(g), x.size,
                                       ctypes.byref(out)))
        return out.value

    def invariants(self, vortices: VortexSystem) -> Invariants:
        x, y, g = self._arrays(vortices)
        out = np.zeros(5)
        self._check(lib.pv_invariants(self._ctx, _ptr(x), _ptr(y), _ptr(g), x.size, _ptr(out)))
        return Invariants.from_array(out)

    # -- device-stepping hooks (src/compute.h:30-36) -------------------------------------------
    def supportsDeviceStepping(self) -> bool:
        return True

    def uploadDeviceState(self, vortices: VortexSystem) -> None:
        x, y, g = self._arrays(vortices)
        self._check(lib.pv_upload_state(self._ctx, _ptr(x), _ptr(y), _ptr(g), x.size))

    def downloadDeviceState(self, vortices: VortexSystem) -> None:
        n = vortices.size()
        x = np.empty(max(n, 1))
        y = np.empty(max(n, 1))
        self._check(lib.pv_download_state(self._ctx, _ptr(x), _ptr(y), n))
        vortices.x = x[:n].copy()
        vortices.y = y[:n].copy()

    def downloadDeviceCirculation(self) -> np.ndarray:
        """Circulations of the device state (they change when dipole events run on it)."""
        n = self.stateSize()
        g = np.empty(max(n, 1))
        self._check(lib.pv_download_circulation(self._ctx, _ptr(g), n))
        return g[:n].copy()

    def downloadDeviceSystem(self) -> VortexSystem:
        """The whole device state (positions and circulations) as a new VortexSystem."""
        g = self.downloadDeviceCirculation()
        s = VortexSystem(np.zeros(g.size), np.zeros(g.size), g)
        self.downloadDeviceState(s)
        return s

    # -- text output formatted on the GPU (the reference's setprecision(17) streams) ----------
    def _formatted(self, call, n_rows: int, row_max: int) -> bytes:
        cap = max(n_rows * row_max, 1)
        buf = ctypes.create_string_buffer(cap)
        length = ctypes.c_size_t(0)
        self._check(call(buf, cap, ctypes.byref(length)))
        return buf.raw[:length.value]

    def formatTrajectory(self, time: float, frame: int) -> bytes:
        """The rows TrajectoryWriter::write (src/print.cpp:29-40) appends for the device state,
        with the velocity evaluated on the device."""
        return self._formatted(lambda b, c, l: lib.pv_format_trajectory(self._ctx, time, frame, b,
                                                                           c, l),
                               self.stateSize(), _lib.TRAJECTORY_ROW_MAX)

    def formatTrajectoryHost(self, time: float, frame: int, vortices: VortexSystem,
                             velocity: VelocityField) -> bytes:
        """The same rows for host arrays."""
        x, y, g = self._arrays(vortices)
        u, v = _f64(velocity.x), _f64(velocity.y)
        if not (u.size == v.size == x.size):
            raise ValueError("velocity and vortex arrays have different lengths")
        return self._formatted(
            lambda b, c, l: lib.pv_format_trajectory_host(self._ctx, time, frame, _ptr(x), _ptr(y),
                                                          _ptr(g), _ptr(u), _ptr(v), x.size, b, c,
                                                          l),
            x.size, _lib.TRAJECTORY_ROW_MAX)

    def formatCheckpointVortices(self) -> bytes:
        """The "x y circulation" block of writeCheckpoint (src/checkpoint.cpp:86-88) for the
        device state."""
        return self._formatted(lambda b, c, l: lib.pv_format_checkpoint_vortices(self._ctx, b, c, l),
                               self.stateSize(), _lib.CHECKPOINT_ROW_MAX)

    def evaluateDeviceState(self) -> VelocityField:
        n = self.stateSize()
        u = np.empty(max(n, 1))
        v = np.empty(max(n, 1))
        self._check(lib.pv_evaluate_state(self._ctx, _ptr(u), _ptr(v), n))
        return VelocityField(u[:n], v[:n])

    def deviceRk4Step(self, dt: float) -> None:
        self._check(lib.pv_rk4_step(self._ctx, dt))

    def deviceDopri5Step(self, dt: float, absoluteTolerance: float, relativeTolerance: float,
                         minimumTimeStep: float, maximumTimeStep: float) -> StepResult:
        r = _lib.PvStepResult()
        self._check(lib.pv_dopri5_step(self._ctx, dt, absoluteTolerance, relativeTolerance,
                                       minimumTimeStep, maximumTimeStep, ctypes.byref(r)))
        return StepResult(r.accepted_time_step, r.suggested_time_step, r.normalized_error,
                          int(r.rejected_steps))

    def invalidateDeviceDerivative(self) -> None:
        self._check(lib.pv_invalidate_derivative(self._ctx))

    # -- additions without a reference counterpart --------------------------------------------
    def stateSize(self) -> int:
        n = ctypes.c_size_t(0)
        self._check(lib.pv_state_size(self._ctx, ctypes.byref(n)))
        return n.value

    def stateInvariants(self) -> Invariants:
        out = np.zeros(5)
        self._check(lib.pv_state_invariants(self._ctx, _ptr(out)))
        return Invariants.from_array(out)

    def dipoleScan(self, threshold: float, capacity: int = 4096) -> list[DipoleCandidate]:
        """Candidates of DipoleManager::process's scan (src/dipole.cpp:49-78) on the device state,
        sorted as the reference sorts them (distance^2, first, second)."""
        while True:
            buf = (_lib.PvDipoleCandidate * max(capacity, 1))()
            count = ctypes.c_size_t(0)
            self._check(lib.pv_dipole_scan(self._ctx, threshold, buf, capacity,
                                           ctypes.byref(count)))
            if count.value <= capacity:
                break
            capacity = count.value
        out = [DipoleCandidate(int(buf[i].first), int(buf[i].second), float(buf[i].distance_squared))
               for i in range(count.value)]
        out.sort(key=lambda c: (c.distanceSquared, c.first, c.second))
        return out

    def statePlan(self) -> dict:
        """How the device state is evaluated (pv_state_plan): symmetric (once per unordered
        pair), partial rows, and the ordered kernel's targets per thread and chunk."""
        info = _lib.PvPlanInfo()
        self._check(lib.pv_state_plan(self._ctx, ctypes.byref(info)))
        return {"symmetric": bool(info.symmetric), "rows": info.rows,
                "targets_per_thread": info.targets_per_thread, "chunk": info.chunk,
                "symmetric_min_ctas": info.symmetric_min_ctas,
                "symmetric_targets": info.symmetric_targets,
                "symmetric_grid_ctas": info.symmetric_grid_ctas}

    @property
    def evaluationCount(self) -> int:
        c = ctypes.c_uint64(0)
        self._check(lib.pv_evaluation_count(self._ctx, ctypes.byref(c)))
        return int(c.value)

    def rk4Advance(self, dt: float, steps: int) -> None:
        self._check(lib.pv_rk4_advance(self._ctx, dt, steps))

    def cudaStream(self) -> int:
        """The context's cudaStream_t as an integer (e.g. for torch.cuda.ExternalStream)."""
        s = ctypes.c_void_p()
        self._check(lib.pv_context_stream(self._ctx, ctypes.byref(s)))
        return int(s.value or 0)

    def setProfiling(self, enabled: bool) -> None:
        """Bracket every kernel launch with CUDA events on the context's stream."""
        self._check(lib.pv_set_profiling(self._ctx, int(bool(enabled))))

    def setNearField(self, radius: float = -1.0) -> None:
        """Near-field radius of the FP32-compensated form (pv_set_near_field): periodic pairs,
        disk pairs and disk wall images closer than it are evaluated in FP64; -1 the default, 0
        none."""
        self._check(lib.pv_set_near_field(self._ctx, float(radius)))

    @property
    def nearField(self) -> float:
        r = ctypes.c_double(0.0)
        self._check(lib.pv_get_near_field(self._ctx, ctypes.byref(r)))
        return float(r.value)

    def setWaitLimits(self, copy_polls: int = -1, barrier_polls: int = -1) -> None:
        """Polls of the bounded device waits before they give up (pv_set_wait_limits): the tile
        copies of a velocity launch and the grid barrier of the cooperative RK4 steps; -1 keeps
        the default, 0 gives up without polling."""
        self._check(lib.pv_set_wait_limits(self._ctx, int(copy_polls), int(barrier_polls)))

    def kernelStats(self) -> dict:
        """{kind: (launches, timed launches, summed milliseconds)} since the last reset."""
        st = _lib.PvKernelStats()
        self._check(lib.pv_get_kernel_stats(self._ctx, ctypes.byref(st)))
        return {k: (int(st.launches[i]), int(st.timed_launches[i]), float(st.milliseconds[i]))
                for i, k in enumerate(_lib.KERNEL_KINDS)}

    def resetKernelStats(self) -> None:
        self._check(lib.pv_reset_kernel_stats(self._ctx))


class InfinitePlaneKernel(VelocityKernel):
    """src/compute.h:37-47."""

    def __init__(self, coreRadius: float = 0.0, **kw):
        super().__init__(_lib.GEOMETRY_INFINITE, core_radius=coreRadius, **kw)


class PeriodicBoxKernel(VelocityKernel):
    """Weiss–McWilliams square torus, src/compute.h:49-62."""

    def __init__(self, lengthX: float, lengthY: float, imageLayers: int = 8, **kw):
        super().__init__(_lib.GEOMETRY_PERIODIC, box_length_x=lengthX, box_length_y=lengthY,
                         image_layers=imageLayers, **kw)


class DiskKernel(VelocityKernel):
    """Circle-theorem images, src/compute.h:63-75."""

    def __init__(self, radius: float, **kw):
        super().__init__(_lib.GEOMETRY_DISK, disk_radius=radius, **kw)


@dataclass
class DipoleEventState:
    """src/dipole.h:12-16."""

    removedPairs: int = 0
    reinjectedPairs: int = 0
    randomEngineState: str = ""


class DeviceDipoleManager:
    """DipoleManager (src/dipole.h:18-40) acting on a kernel's device-resident state.

    process() is DipoleManager::process (src/dipole.cpp:42-127) with the candidate scan and the
    survivor compaction on the GPU; only the candidate list crosses to the host, where the
    closest-first selection and the reinjection draws (the reference's generator, seeded as the
    reference seeds it) are made. After it the device population, its order and the generator
    state equal what the reference's host code leaves. `state` restores a checkpointed
    DipoleEventState (src/dipole.cpp:32-40)."""

    def __init__(self, kernel: "VelocityKernel", removal: bool = True, distance: float = 0.01,
                 reinjection: str = "none", random_seed: int = 1234567,
                 state: Optional[DipoleEventState] = None):
        if reinjection not in _lib.REINJECTION:
            raise ValueError("dipoleReinjection must be none, independent, or paired")
        self.kernel = kernel
        cfg = _lib.PvDipoleConfig(int(bool(removal)), float(distance),
                                  _lib.REINJECTION[reinjection], int(random_seed) & (2**64 - 1))
        kernel._check(lib.pv_dipole_configure(kernel._ctx, ctypes.byref(cfg)))
        if state is not None:
            kernel._check(lib.pv_dipole_restore(kernel._ctx, state.removedPairs,
                                                state.reinjectedPairs,
                                                state.randomEngineState.encode()))

    def process(self) -> int:
        events = ctypes.c_size_t(0)
        self.kernel._check(lib.pv_dipole_process(self.kernel._ctx, ctypes.byref(events)))
        return int(events.value)

    def state(self) -> DipoleEventState:
        removed, reinjected = ctypes.c_uint64(0), ctypes.c_uint64(0)
        length = ctypes.c_size_t(0)
        lib.pv_dipole_state(self.kernel._ctx, ctypes.byref(removed), ctypes.byref(reinjected),
                            None, 0, ctypes.byref(length))
        buf = ctypes.create_string_buffer(length.value + 1)
        self.kernel._check(lib.pv_dipole_state(self.kernel._ctx, ctypes.byref(removed),
                                               ctypes.byref(reinjected), buf, len(buf),
                                               ctypes.byref(length)))
        return DipoleEventState(int(removed.value), int(reinjected.value), buf.value.decode())


def computeInvariants(vortices: VortexSystem, kernel: VelocityKernel) -> Invariants:
    """computeInvariants(vortices, kernel), src/compute.cpp:157-163, on the GPU."""
    return kernel.invariants(vortices)


def makeBackendKernel(params: dict) -> VelocityKernel:
    """makeBackendKernel(SimParams) (src/backend.h:16; makeReferenceKernel,
    src/backend_common.cpp:4-13). ``params`` uses the parameter-file keys."""
    bc = params.get("boundaryCondition", "infinite")
    precision = params.get("precision", _lib.PRECISION_FP64)
    if bc == "infinite":
        return InfinitePlaneKernel(params.get("coreRadius", 0.0), precision=precision)
    if bc == "periodic":
        return PeriodicBoxKernel(params.get("boxLengthX", 2.0), params.get("boxLengthY", 2.0),
                                 params.get("periodicImageLayers", 8), precision=precision)
    if bc == "disk":
        return DiskKernel(params.get("diskRadius", 1.0), precision=precision)
    raise ValueError("unsupported boundary condition: " + str(bc))


def backendName() -> str:
    return lib.pv_backend_name().decode()


def backendRuntimeDetails(device: int = 0) -> str:
    buf = ctypes.create_string_buffer(512)
    rc = lib.pv_runtime_details(device, buf, len(buf))
    if rc != _lib.PV_OK:
        raise CudaError(lib.pv_last_error(None).decode())
    return buf.value.decode()


def probePeak(kind: str = "fp64", device: int = 0) -> float:
    """Measured FMA throughput of the GPU in FLOP/s (kind "fp64" or "fp32")."""
    out = ctypes.c_double(0.0)
    rc = lib.pv_probe_peak(device, 0 if kind == "fp64" else 1, ctypes.byref(out))
    if rc != _lib.PV_OK:
        raise CudaError(lib.pv_last_error(None).decode())
    return out.value
