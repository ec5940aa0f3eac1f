"""Autotuner of the velocity plan: for every geometry, precision and N bucket (floor(log2 N)) it
times the tiled kernel with 1, 2 and 4 targets per thread on a seeded state of that size and keeps
the fastest in the library's tuning table (pv_set_tuning). Results are cached as JSON; the package
loads `tuning.json` next to this file when it exists.

    python -m pointvortex_b200.autotune [--out path] [--min-log2 6] [--max-log2 16]
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


def load(path: str = DEFAULT_PATH) -> int:
    """Applies a cached table; returns the number of entries."""
    if not os.path.exists(path):
        return 0
    with open(path) as f:
        table = json.load(f)
    for e in table.get("entries", []):
        set_entry(GEOMETRIES[e["geometry"]], PRECISIONS[e["precision"]], e["log2_n"], e["per_thread"])
    return len(table.get("entries", []))


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
    return {"entries": entries}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=DEFAULT_PATH)
    ap.add_argument("--min-log2", type=int, default=6)
    ap.add_argument("--max-log2", type=int, default=16)
    ap.add_argument("--evals", type=int, default=3)
    args = ap.parse_args(argv)
    table = tune(log2_range=range(args.min_log2, args.max_log2 + 1), evals=args.evals)
    with open(args.out, "w") as f:
        json.dump(table, f, indent=1)
    print(f"wrote {len(table['entries'])} entries to {args.out}")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
