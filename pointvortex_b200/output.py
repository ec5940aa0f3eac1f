"""Trajectory and checkpoint files in the reference's formats, with the per-vortex text made on
the GPU.

The reference writes every number with `std::ostream << std::setprecision(17)` (src/print.cpp:20,
src/checkpoint.cpp:41): 17 significant digits, correctly rounded, "%g" layout. For large N and
frequent output that host formatting dominates a run. Here the per-vortex rows are formatted by
libpvb200 on the GPU, byte-identical, and cross to the host as one block of text; only the few
header numbers of a checkpoint are formatted on the host (Python's "%.17g" is correctly rounded
like the C library's).
"""
from __future__ import annotations

import math
import os
import struct
from dataclasses import dataclass
from typing import Optional, Sequence

from .kernel import DipoleEventState, Invariants, VelocityField, VelocityKernel, VortexSystem

TRAJECTORY_HEADER = b"time,frame,index,x,y,circulation,u,v\n"
CHECKPOINT_MAGIC = "POINT_VORTEX_CHECKPOINT"
CHECKPOINT_VERSION = 6


def g17(v: float) -> str:
    """One double as the reference's streams print it (C's "%.17g"; glibc prints a NaN with its
    sign)."""
    v = float(v)
    if math.isnan(v):
        return "-nan" if struct.pack(">d", v)[0] & 0x80 else "nan"
    return "%.17g" % v


def _open_output(filename: str, overwrite: bool, description: str):
    """openOutput (src/print.cpp:9-21)."""
    if not overwrite and os.path.exists(filename):
        raise RuntimeError(f"refusing to overwrite {description}: {filename}")
    parent = os.path.dirname(filename)
    if parent:
        os.makedirs(parent, exist_ok=True)
    try:
        return open(filename, "wb")
    except OSError as exc:
        raise RuntimeError(f"cannot open {description}: {filename}") from exc


class TrajectoryWriter:
    """TrajectoryWriter (src/print.h:8-16, src/print.cpp:24-40). `kernel` is the context whose
    GPU formats the rows (any VelocityKernel of this package)."""

    def __init__(self, filename: str, overwrite: bool, kernel: VelocityKernel):
        self.kernel = kernel
        self._out = _open_output(filename, overwrite, "output file")
        self._out.write(TRAJECTORY_HEADER)
        self._out.flush()

    def write(self, time: float, frame: int, vortices: VortexSystem, velocity: VelocityField):
        """One frame from host arrays (the reference's signature)."""
        self._emit(self.kernel.formatTrajectoryHost(time, frame, vortices, velocity))

    def write_device_state(self, time: float, frame: int):
        """One frame of the kernel's device state, the velocity evaluated on the device: the
        driver's writeTrajectory (src/main.cpp:251-258) without downloading the state."""
        self._emit(self.kernel.formatTrajectory(time, frame))

    def _emit(self, rows: bytes):
        try:
            self._out.write(rows)
            self._out.flush()
        except OSError as exc:
            raise RuntimeError("failed while writing trajectory output") from exc

    def close(self):
        self._out.close()


@dataclass
class OutputSchedule:
    """src/checkpoint.h:9-15."""

    trajectoryInterval: float = 0.0
    diagnosticsInterval: float = 0.0
    checkpointInterval: float = 0.0
    nextDiagnosticsTime: float = 0.0
    nextCheckpointTime: float = 0.0


@dataclass
class CheckpointProgress:
    """src/checkpoint.h:16-23."""

    time: float
    suggestedTimeStep: float
    nextOutputTime: float
    acceptedSteps: int
    outputIndex: int
    eventIndex: int


def checkpoint_path(directory: str, output_index: int) -> str:
    """checkpointPath (src/checkpoint.cpp:17-22)."""
    return os.path.join(directory, "checkpoint_%08d.dat" % output_index)


def _invariants(v) -> Sequence[float]:
    if isinstance(v, Invariants):
        return (v.circulation, v.linearImpulseX, v.linearImpulseY, v.angularImpulse, v.hamiltonian)
    return tuple(v)


def checkpoint_header(n: int, initial, params: dict, segment, dipole_state: DipoleEventState,
                      schedule: OutputSchedule, progress: CheckpointProgress) -> bytes:
    """The lines writeCheckpoint (src/checkpoint.cpp:42-85) writes before the vortex block.
    `params` uses the parameter-file keys (boundaryCondition, coreRadius, boxLengthX, boxLengthY,
    diskRadius, periodicImageLayers, integrator, dipoleRemoval, dipoleRemovalDistance,
    dipoleReinjection)."""
    bc = params.get("boundaryCondition", "infinite")
    gx = (params.get("boxLengthX", 2.0) if bc == "periodic"
          else params.get("diskRadius", 1.0) if bc == "disk" else 0.0)
    gy = params.get("boxLengthY", 2.0) if bc == "periodic" else 0.0
    layers = int(params.get("periodicImageLayers", 8)) if bc == "periodic" else 0
    s = schedule
    lines = [
        f"{CHECKPOINT_MAGIC} {CHECKPOINT_VERSION}",
        f"time {g17(progress.time)}",
        f"suggested_time_step {g17(progress.suggestedTimeStep)}",
        f"next_output_time {g17(progress.nextOutputTime)}",
        "output_schedule " + " ".join(g17(v) for v in (
            s.trajectoryInterval, s.diagnosticsInterval, s.checkpointInterval,
            s.nextDiagnosticsTime, s.nextCheckpointTime)),
        f"accepted_steps {int(progress.acceptedSteps)}",
        f"output_index {int(progress.outputIndex)}",
        f"event_index {int(progress.eventIndex)}",
        f"core_radius {g17(params.get('coreRadius', 0.0))}",
        f"integrator {params.get('integrator', 'dopri5')}",
        f"geometry {bc} {g17(gx)} {g17(gy)} {layers}",
        f"dipole_config {int(bool(params.get('dipoleRemoval', False)))} "
        f"{g17(params.get('dipoleRemovalDistance', 0.01))} "
        f"{params.get('dipoleReinjection', 'none')}",
        f"dipole_counts {int(dipole_state.removedPairs)} {int(dipole_state.reinjectedPairs)}",
        f"random_engine_state {dipole_state.randomEngineState}",
        "initial_invariants " + " ".join(g17(v) for v in _invariants(initial)),
        "segment_invariants " + " ".join(g17(v) for v in _invariants(segment)),
        f"vortex_count {n}",
        "vortices",
    ]
    return ("\n".join(lines) + "\n").encode()


def write_checkpoint(directory: str, kernel: VelocityKernel, initial, params: dict, segment,
                     dipole_state: Optional[DipoleEventState], schedule: OutputSchedule,
                     progress: CheckpointProgress, overwrite: bool = False) -> str:
    """writeCheckpoint (src/checkpoint.cpp:23-102) of the kernel's device state: the vortex
    block is formatted on the GPU. The file appears atomically (temporary file, fsync, rename,
    directory fsync). Returns the checkpoint's path."""
    dipole_state = dipole_state or DipoleEventState()
    os.makedirs(directory, exist_ok=True)
    destination = checkpoint_path(directory, progress.outputIndex)
    if not overwrite and os.path.exists(destination):
        raise RuntimeError("refusing to overwrite checkpoint: " + destination)
    temporary = destination + ".tmp"
    body = kernel.formatCheckpointVortices()
    header = checkpoint_header(kernel.stateSize(), initial, params, segment, dipole_state,
                               schedule, progress)
    try:
        with open(temporary, "wb") as f:
            f.write(header)
            f.write(body)
            f.flush()
            os.fsync(f.fileno())
    except OSError as exc:
        raise RuntimeError("failed while writing checkpoint: " + temporary) from exc
    os.replace(temporary, destination)
    try:
        fd = os.open(directory, os.O_RDONLY | getattr(os, "O_DIRECTORY", 0))
        try:
            os.fsync(fd)
        finally:
            os.close(fd)
    except OSError:
        pass
    return destination
