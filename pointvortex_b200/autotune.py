"""Autotuner of the velocity plans, per geometry, precision and N bucket (floor(log2 N)), on a
seeded state of that size, keeping the fastest in the library's tables:

* the ordered-pair kernel: 1, 2 or 4 targets per thread (pv_set_tuning);
* the once-per-unordered-pair form of the periodic box and the plane (pv_set_symmetric_tuning):
  the ordered kernel or the symmetric form, and for the symmetric form the occupancy it is built
  for (periodic FP64: the default, 7 or 8 CTAs per SM) or the targets per lane (plane: 4 or 8).
  A candidate is timed per evaluation inside DOPRI5 steps of the device state (velocity launches,
  stage kernels, the captured attempt), the way the steppers use it;
* for the chosen symmetric form, the persistent grid's CTAs per SM (pv_set_symmetric_grid): as
  many as fit, or down to three fewer (a fuller last round of the work queue can finish sooner);
* the batch engine's ordered work items: 1, 2 or 4 targets per thread (pv_set_batch_tuning),
  timed per DOPRI5 attempt of a batch of simulations of that size (as many as make about 2^26
  pair interactions per evaluation, at most 512), so the choice is made where the grid is full.

Results are cached as JSON; the package loads `tuning.json` next to this file when it exists.

    python -m pointvortex_b200.autotune [--out path] [--min-log2 6] [--max-log2 16]
    python -m pointvortex_b200.autotune --only batch [--out path]   # replace the batch part only
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os

from . import _lib, ics
from ._lib import lib

DEFAULT_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning.json")
GEOMETRIES = {"infinite": 0, "periodic": 1, "disk": 2}
PRECISIONS = {"fp64": 0, "fp32c": 1}


def set_entry(geometry: int, precision: int, log2_n: int, per_thread: int) -> None:
    rc = lib.pv_set_tuning(geometry, precision, log2_n, per_thread)
    if rc != _lib.PV_OK:
        raise ValueError(lib.pv_last_error(None).decode())


def get_entry(geometry: int, precision: int, log2_n: int) -> int:
    out = ctypes.c_int(0)
    lib.pv_get_tuning(geometry, precision, log2_n, ctypes.byref(out))
    return out.value


def set_symmetric_entry(geometry: int, precision: int, log2_n: int, mode: int, min_ctas: int = 0,
                        targets: int = 0) -> None:
    rc = lib.pv_set_symmetric_tuning(geometry, precision, log2_n, mode, min_ctas, targets)
    if rc != _lib.PV_OK:
        raise ValueError(lib.pv_last_error(None).decode())


def get_symmetric_entry(geometry: int, precision: int, log2_n: int) -> tuple:
    m, c, t = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0)
    lib.pv_get_symmetric_tuning(geometry, precision, log2_n, ctypes.byref(m), ctypes.byref(c),
                                ctypes.byref(t))
    return m.value, c.value, t.value


def set_symmetric_grid(geometry: int, precision: int, log2_n: int, ctas_per_sm: int) -> None:
    rc = lib.pv_set_symmetric_grid(geometry, precision, log2_n, ctas_per_sm)
    if rc != _lib.PV_OK:
        raise ValueError(lib.pv_last_error(None).decode())


def get_symmetric_grid(geometry: int, precision: int, log2_n: int) -> int:
    out = ctypes.c_int(0)
    lib.pv_get_symmetric_grid(geometry, precision, log2_n, ctypes.byref(out))
    return out.value


def set_batch_entry(geometry: int, precision: int, log2_n: int, per_thread: int) -> None:
    rc = lib.pv_set_batch_tuning(geometry, precision, log2_n, per_thread)
    if rc != _lib.PV_OK:
        raise ValueError(lib.pv_last_error(None).decode())


def get_batch_entry(geometry: int, precision: int, log2_n: int) -> int:
    out = ctypes.c_int(0)
    lib.pv_get_batch_tuning(geometry, precision, log2_n, ctypes.byref(out))
    return out.value


def load(path: str = DEFAULT_PATH) -> int:
    """Applies a cached table; returns the number of entries."""
    if not os.path.exists(path):
        return 0
    with open(path) as f:
        table = json.load(f)
    for e in table.get("entries", []):
        set_entry(GEOMETRIES[e["geometry"]], PRECISIONS[e["precision"]], e["log2_n"], e["per_thread"])
    for e in table.get("symmetric", []):
        set_symmetric_entry(GEOMETRIES[e["geometry"]], PRECISIONS[e["precision"]], e["log2_n"],
                            e["mode"], e.get("min_ctas", 0), e.get("targets", 0))
        set_symmetric_grid(GEOMETRIES[e["geometry"]], PRECISIONS[e["precision"]], e["log2_n"],
                           e.get("grid_ctas", 0))
    for e in table.get("batch", []):
        set_batch_entry(GEOMETRIES[e["geometry"]], PRECISIONS[e["precision"]], e["log2_n"],
                        e["per_thread"])
    return sum(len(table.get(k, [])) for k in ("entries", "symmetric", "batch"))


def _time_plan(geometry: str, precision: int, n: int, per_thread: int, evals: int) -> float:
    from .kernel import DiskKernel, InfinitePlaneKernel, PeriodicBoxKernel, VortexSystem
    set_entry(GEOMETRIES[geometry], precision, n.bit_length() - 1, per_thread)
    if geometry == "infinite":
        k = InfinitePlaneKernel(0.0, precision=precision)
        x, y, g = ics.infinite_plane(n, 1)
    elif geometry == "periodic":
        k = PeriodicBoxKernel(6.283185307179586, 6.283185307179586, 8, precision=precision)
        x, y, g = ics.periodic_box(n + n % 2, 1)
    else:
        k = DiskKernel(1.0, precision=precision)
        x, y, g = ics.disk(n, 1)
    k.uploadDeviceState(VortexSystem(x, y, g))
    k.evaluateDeviceState()
    k.setProfiling(True)
    k.resetKernelStats()
    for _ in range(evals):
        k.evaluateDeviceState()
    _, timed, ms = k.kernelStats()["velocity"]
    k.close()
    return ms / max(timed, 1)


def _time_steps(geometry: str, precision: int, n: int, steps: int) -> float:
    """ms per evaluation inside DOPRI5 steps of the device state (the captured attempt with its
    stage kernels and programmatic launches, as the steppers run it), current tables. An
    evaluation timed alone can rank plans differently: a grid that leaves SM room lets the next
    kernels of a step start early beside it."""
    import time
    from .kernel import InfinitePlaneKernel, PeriodicBoxKernel, VortexSystem
    if geometry == "infinite":
        k = InfinitePlaneKernel(0.0, precision=precision)
        x, y, g = ics.infinite_plane(n, 1)
    else:
        k = PeriodicBoxKernel(6.283185307179586, 6.283185307179586, 8, precision=precision)
        x, y, g = ics.periodic_box(n + n % 2, 1)
    k.uploadDeviceState(VortexSystem(x, y, g))
    dt = 1e-3
    for _ in range(3):
        dt = k.deviceDopri5Step(dt, 1e-12, 1e-9, 1e-12, 0.1).suggestedTimeStep
    e0 = k.evaluationCount
    t0 = time.perf_counter()
    for _ in range(steps):
        dt = k.deviceDopri5Step(dt, 1e-12, 1e-9, 1e-12, 0.1).suggestedTimeStep
    t1 = time.perf_counter()
    evals = k.evaluationCount - e0
    k.close()
    return (t1 - t0) * 1e3 / max(evals, 1)


# candidates of the symmetric-form table: (mode, min_ctas, targets)
SYMMETRIC_CANDIDATES = {
    ("periodic", "fp64"): [(1, 0, 0), (2, 0, 0), (2, 7, 0), (2, 8, 0), (2, 0, 2)],
    ("periodic", "fp32c"): [(1, 0, 0), (2, 0, 0)],
    ("infinite", "fp64"): [(1, 0, 0), (2, 0, 4), (2, 0, 8)],
    ("infinite", "fp32c"): [(1, 0, 0), (2, 0, 4), (2, 0, 8)],
}


def tune_symmetric(log2_range=range(11, 17), evals: int = 3) -> list:
    """Each candidate timed per evaluation inside DOPRI5 steps (_time_steps), 3 + evals steps."""
    entries = []
    steps = max(evals, 3)
    for (geo, prec), cands in SYMMETRIC_CANDIDATES.items():
        for b in log2_range:
            n = 1 << b
            times = {}
            for cand in cands:
                set_symmetric_entry(GEOMETRIES[geo], PRECISIONS[prec], b, *cand)
                times[cand] = _time_steps(geo, PRECISIONS[prec], n, steps)
            best = min(times, key=times.get)
            set_symmetric_entry(GEOMETRIES[geo], PRECISIONS[prec], b, *best)
            grid, grid_ms = 0, {}
            if best[0] == 2:
                set_symmetric_grid(GEOMETRIES[geo], PRECISIONS[prec], b, 0)
                fit = _grid_ctas(geo, PRECISIONS[prec], n)
                grid_ms[fit] = times[best]
                for c in range(fit - 1, max(fit - 4, 1), -1):
                    set_symmetric_grid(GEOMETRIES[geo], PRECISIONS[prec], b, c)
                    grid_ms[c] = _time_steps(geo, PRECISIONS[prec], n, steps)
                best_c = min(grid_ms, key=grid_ms.get)
                grid = 0 if best_c == fit else best_c
            set_symmetric_grid(GEOMETRIES[geo], PRECISIONS[prec], b, grid)
            entries.append({"geometry": geo, "precision": prec, "log2_n": b, "mode": best[0],
                            "min_ctas": best[1], "targets": best[2], "grid_ctas": grid,
                            "ms": {"/".join(map(str, c)): v for c, v in times.items()},
                            "grid_ms": {str(c): v for c, v in grid_ms.items()}})
    return entries


def _grid_ctas(geometry: str, precision: int, n: int) -> int:
    """CTAs per SM of the symmetric form's grid as the current tables plan it."""
    from .kernel import InfinitePlaneKernel, PeriodicBoxKernel, VortexSystem
    if geometry == "infinite":
        k = InfinitePlaneKernel(0.0, precision=precision)
        x, y, g = ics.infinite_plane(n, 1)
    else:
        k = PeriodicBoxKernel(6.283185307179586, 6.283185307179586, 8, precision=precision)
        x, y, g = ics.periodic_box(n + n % 2, 1)
    k.uploadDeviceState(VortexSystem(x, y, g))
    c = k.statePlan()["symmetric_grid_ctas"]
    k.close()
    return c


# targets per thread of the batch's ordered items, by geometry (pv_set_batch_tuning allows these)
BATCH_CANDIDATES = {"infinite": (1, 2, 4), "periodic": (1, 2), "disk": (1, 2, 4)}


def batch_room(n: int) -> tuple:
    """(simulations, arena vortices, partial chunks per vortex slot) of the tuner's batch of
    population n: as many simulations as make about 2^26 pair interactions per evaluation (at
    most 512), each with room for the most partial rows a simulation of that size can take: one
    per 128-block in the once-per-unordered-pair form, else one per source chunk (at most 33)."""
    sims = max(1, min(512, (1 << 26) // (n * n)))
    return sims, sims * (n + 256) + 256, max(-(-n // 128), 64) + 1


def _time_batch(geometry: str, precision: str, n: int, attempts: int) -> float | None:
    """ms per DOPRI5 attempt of a batch of equal simulations of population n under the current
    batch table, or None where the simulations take the once-per-unordered-pair items (the table
    does not apply). Two untimed attempts first; the simulations run far from their end time."""
    import time
    from .batch import Batch, geometry_params
    sims, vortices, chunks = batch_room(n)
    b = Batch(vortices, sims, max_steps=1 << 30, partial_factor=chunks)
    try:
        for s in range(sims):
            if geometry == "periodic":
                st = ics.periodic_box(n + n % 2, 100 + s)
            elif geometry == "disk":
                st = ics.disk(n, 100 + s, 1.0, 0.95, gaussian=False)
            else:
                st = ics.infinite_plane(n, 100 + s)
            sid = b.add(geometry_params(geometry, precision=precision), *st, 1e6, dt=1e-4,
                        atol=1e-10, rtol=1e-8)
            if b.info(sid).targetsPerThread == 0:
                return None
        b.advance(2)
        t0 = time.perf_counter()
        b.advance(attempts)
        return (time.perf_counter() - t0) * 1e3 / attempts
    finally:
        b.close()


def tune_batch(log2_range=range(5, 16), attempts: int = 6) -> list:
    """Each candidate of BATCH_CANDIDATES timed per attempt (_time_batch); the fastest is kept.
    A size whose batch cannot be admitted (CapacityError: the device's memory) keeps the default
    and is reported on stderr; the other sizes are still tuned."""
    import sys
    from .batch import CapacityError
    entries = []
    for geo, cands in BATCH_CANDIDATES.items():
        for prec in PRECISIONS:
            for b in log2_range:
                times = {}
                for t in cands:
                    set_batch_entry(GEOMETRIES[geo], PRECISIONS[prec], b, t)
                    try:
                        ms = _time_batch(geo, prec, 1 << b, attempts)
                    except CapacityError as exc:
                        print(f"batch tuning: {geo} {prec} N = 2^{b} skipped: {exc}",
                              file=sys.stderr)
                        times = {}
                        break
                    if ms is None:
                        break
                    times[t] = ms
                if not times:
                    set_batch_entry(GEOMETRIES[geo], PRECISIONS[prec], b, 0)
                    continue
                best = min(times, key=times.get)
                set_batch_entry(GEOMETRIES[geo], PRECISIONS[prec], b, best)
                entries.append({"geometry": geo, "precision": prec, "log2_n": b, "per_thread": best,
                                "ms": {str(k): v for k, v in times.items()}})
    return entries


def tune(geometries=("infinite", "periodic", "disk"), precisions=("fp64", "fp32c"),
         log2_range=range(6, 17), evals: int = 3) -> dict:
    entries = []
    for geo in geometries:
        for prec in precisions:
            for b in log2_range:
                n = 1 << b
                times = {t: _time_plan(geo, PRECISIONS[prec], n, t, evals) for t in (1, 2, 4)}
                best = min(times, key=times.get)
                set_entry(GEOMETRIES[geo], PRECISIONS[prec], b, best)
                entries.append({"geometry": geo, "precision": prec, "log2_n": b, "per_thread": best,
                                "ms": {str(k): v for k, v in times.items()}})
    symmetric = tune_symmetric(range(max(11, log2_range.start), log2_range.stop), evals)
    batch = tune_batch(range(max(5, log2_range.start - 1), min(16, log2_range.stop)))
    return {"entries": entries, "symmetric": symmetric, "batch": batch}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=DEFAULT_PATH)
    ap.add_argument("--min-log2", type=int, default=6)
    ap.add_argument("--max-log2", type=int, default=16)
    ap.add_argument("--evals", type=int, default=3)
    ap.add_argument("--only", choices=["batch"], default=None,
                    help="tune only the batch table, keeping the rest of the table at --out")
    args = ap.parse_args(argv)
    if args.only == "batch":
        table = {}
        if os.path.exists(args.out):
            with open(args.out) as f:
                table = json.load(f)
        load(args.out)
        table["batch"] = tune_batch()
    else:
        table = tune(log2_range=range(args.min_log2, args.max_log2 + 1), evals=args.evals)
    with open(args.out, "w") as f:
        json.dump(table, f, indent=1)
    print(f"wrote {sum(len(table.get(k, [])) for k in ('entries', 'symmetric', 'batch'))} "
          f"entries to {args.out}")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
