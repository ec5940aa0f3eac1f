"""Builds libpvb200.so in-tree with nvcc for sm_100a.

    python pointvortex_b200/build.py           # build if any source is newer than the library
    python pointvortex_b200/build.py --force   # rebuild

The library is written to pointvortex_b200/libpvb200.so, next to this file, so that it travels
with the source tree and is the one the package loads.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libpvb200.so")
OBJ_DIR = os.path.join(HERE, "_build")
SOURCES = ["pv_velocity.cu", "pv_velocity32.cu", "pv_stepping.cu", "pv_invariants.cu", "pv_dipole.cu", "pv_context.cu",
           "pv_noalloc.cu", "pv_batch.cu", "pv_output.cu", "pv_symmetric.cu", "pv_near.cu"]
HEADERS = ["pv_common.cuh", "pv_geometry.cuh", "pv_format.cuh", "pv_pair32.cuh", "pv_symmetric.cuh",
           "pv_internal.h"]
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC,-O2",
    "--expt-relaxed-constexpr",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    """Compile every CUDA source of the library and link libpvb200.so; returns its path."""
    os.makedirs(OBJ_DIR, exist_ok=True)
    nvcc = _nvcc()
    include = ["-I", os.path.join(ROOT, "include"), "-I", CSRC]
    headers = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "pvb200.h")]
    objects = []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(OBJ_DIR, src.replace(".cu", ".o"))
        objects.append(obj)
        if force or _newer(obj, [path] + headers + [__file__]):
            cmd = [nvcc, *NVCC_FLAGS, *include, "-c", path, "-o", obj]
            if ptxas_info:
                cmd.insert(1, "-Xptxas=-v")
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if force or _newer(LIB, objects):
        cmd = [nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objects, "-o", LIB,
               "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true")
    args = ap.parse_args(argv)
    print(build(force=args.force, verbose=args.verbose, ptxas_info=args.ptxas_info))
    return 0


if __name__ == "__main__":
    sys.exit(main())
