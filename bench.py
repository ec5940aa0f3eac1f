"""Benchmark of the B200 point-vortex path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one GPU): the periodic-box case -- N = 4096 vortices, uniform in the 2 pi box, balanced
+-1 circulations, Weiss-McWilliams kernel with M = 8 image layers, adaptive DOPRI5 with
rtol 1e-9 / atol 1e-12, close-dipole detection at separation 1e-3 (removal only) after every
accepted step. One step = one accepted DOPRI5 step (with its rejections, 6 velocity evaluations
per attempt thanks to FSAL) plus the dipole scan. The metric is pair-interactions per second,
N(N-1) per velocity evaluation.

With --gpus N (launched one process per GPU) every rank runs its own independent simulation
(replicas: the path has no data exchange), and the value is the total over ranks.

--impl reference times the reference's own CPU implementation (the unmodified PointVortex code
compiled from its sources into oracle/_ref) on the same workload and metric, with all host
threads: its own DOPRI5 steps and dipole events, timed for as many of the K steps as fit a
bounded wall-clock budget. That arm never imports the package (no libpvb200.so is mapped).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N = 4096
LENGTH = 2.0 * np.pi
LAYERS = 8
RTOL, ATOL, DTMIN, DTMAX, DT0 = 1e-9, 1e-12, 1e-12, 0.1, 1e-3
DIPOLE_THRESHOLD = 1e-3
SEED = 20240102
WORKLOAD = "periodic_dopri5_n4096"
L2_BYTES = 126 * 1024 * 1024
METRIC = "pair-interactions/s"

# Algorithmic FP64 operations per ordered pair of the periodic evaluation (FMA = 2, add/mul/
# reciprocal/rint = 1), as the truncated image series is evaluated (pv_geometry.cuh,
# PeriodicPair): per axis the displacement, exact remainder and scaling (7) and the shared
# sinh/cosh/sin/cos Taylor series of the half angle (48); the derived cosh, cos, sin, sinh of the
# full angles (20) and the two m = 0 denominators (8); per axis the image sum -- setup (6), the
# exact m = +-1, +-2 pairs (18), the m = 3..5 expansion (6) and the m = +-6 terms (5); per axis
# the combination, reciprocal and update (16).
FLOPS_PER_PAIR_PERIODIC = 240
# The symmetric form evaluates each unordered pair once and applies it to both vortices: the same
# 240 plus two more FMA updates (the source's reaction) per unordered pair.
FLOPS_PER_UNORDERED_PAIR_SYMMETRIC = 244
# The work these counts state is kept fixed, so that the roofline fraction stays comparable as the
# kernel changes. What the kernel now executes per unordered pair is less (economized series,
# shared doubled values, the m = 1, 2 fraction started from m = 1, the m = +-6 images in the
# m = 3..6 expansion): 189, counted by ncu as 2 x DFMA + DMUL + DADD per unordered pair (72.5,
# 36.3 and 8.1 FP64 instructions) at N = 4096.
FLOPS_EXECUTED_PER_UNORDERED_PAIR_SYMMETRIC = 189
# The plane in the same count: an ordered pair is 11 (displacement 2, r^2 3, reciprocal 1, scale
# 1, two FMA updates 4); the symmetric form spends 16 per unordered pair (the shared displacement,
# r^2 and reciprocal, the two kernel values 2, four FMA updates 8).
FLOPS_PER_PAIR_PLANE = 11
FLOPS_PER_UNORDERED_PAIR_PLANE_SYMMETRIC = 16
# DRAM bytes (read + write) of one launch of the symmetric periodic kernel at this workload, from
# one ncu capture (dram__bytes_read.sum 174.8 KB, dram__bytes_write.sum 0 B, with ncu's cache
# flush before the launch): the sources are read once, the partial rows stay in L2.
TRAFFIC_BYTES_PER_LAUNCH = 174848


def load_ics():
    """The seeded IC generator (pointvortex_b200/ics.py, plain numpy), loaded from its file. The
    reference arm, the CPU baselines and the reference CUDA leg use it this way so that they never
    import the package, whose import maps libpvb200.so."""
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "pvb200_ics_standalone", os.path.join(ROOT, "pointvortex_b200", "ics.py"))
    module = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(module)
    return module


def rank_info():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.rows = []
        self._stop = threading.Event()
        self._thread = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.device),
                                      f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits"],
                                     capture_output=True, text=True, timeout=5).stdout.strip()
                if out:
                    self.rows.append([c.strip() for c in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._thread = threading.Thread(target=self._run, daemon=True)
        self._thread.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._thread:
            self._thread.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4)
                          if len(r) > 5 + k and r[5 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def combine_ranks(total_ms: float, pairs: float, device: str = "cpu"):
    """Whole-job figures of the replicas: the slowest rank's device time (max) and the pairs all
    ranks evaluated (sum). Without a process group it returns its inputs."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return total_ms, pairs
    t = torch.tensor([total_ms], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    p = torch.tensor([pairs], device=device, dtype=torch.float64)
    dist.all_reduce(p)
    return float(t.item()), float(p.item())


def flush_l2(buf):
    buf.fill_(1.0)


def dopri_step(k, dt, dipoles=None):
    """One accepted DOPRI5 step + the close-dipole events (removal only) on the device state;
    returns (suggested dt, evaluations)."""
    before = k.evaluationCount
    r = k.deviceDopri5Step(dt, ATOL, RTOL, DTMIN, DTMAX)
    if dipoles is not None:
        dipoles.process()
    return r.suggestedTimeStep, k.evaluationCount - before


def dipole_manager(k, seed):
    """DipoleManager of the workload (removal only, src/dipole.cpp:42-127) on the device state:
    the scan runs on the GPU and, when it finds pairs, only the candidates reach the host."""
    import pointvortex_b200 as pv
    return pv.DeviceDipoleManager(k, removal=True, distance=DIPOLE_THRESHOLD, reinjection="none",
                                  random_seed=seed)


def run_ours(args):
    import torch
    import pointvortex_b200 as pv
    from pointvortex_b200 import ics

    rank, world, local = rank_info()
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", device_id=torch.device("cuda", local),
                                timeout=__import__("datetime").timedelta(seconds=120))
    x, y, g = ics.periodic_box(N, SEED + rank, LENGTH)
    k = pv.PeriodicBoxKernel(LENGTH, LENGTH, LAYERS, device=local)
    k.uploadDeviceState(pv.VortexSystem(x, y, g))
    dipoles = dipole_manager(k, SEED + rank)
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=f"cuda:{local}")

    # warm-up: the first steps also absorb the start-up rejections (dt 1e-3 -> ~1e-6)
    dt = DT0
    for _ in range(max(args.warmup, 3)):
        dt, _ = dopri_step(k, dt, dipoles)
    torch.cuda.synchronize()

    # timed region: CUDA events on the library's own stream bracket each step (kernels, copies
    # and the gaps while the host reads the step-control word back)
    k.setProfiling(False)
    k.resetKernelStats()
    lib_stream = torch.cuda.ExternalStream(k.cudaStream(), device=f"cuda:{local}")

    def run_steps(dt, record):
        evals, pairs = 0, 0.0
        events = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                  for _ in range(args.steps)] if record else None
        for s in range(args.steps):
            flush_l2(flush)
            torch.cuda.synchronize()
            n_step = k.stateSize()       # the evaluations of a step run before its removals
            if record:
                events[s][0].record(lib_stream)
            dt, e = dopri_step(k, dt, dipoles)
            if record:
                events[s][1].record(lib_stream)
            evals += e
            pairs += e * n_step * (n_step - 1)
        torch.cuda.synchronize()
        step_ms = [a.elapsed_time(b) for a, b in events] if record else None
        return dt, evals, pairs, step_ms

    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        dt, evals, pairs, step_ms = run_steps(dt, True)
        launches = sum(v[0] for v in k.kernelStats().values())
        # kernel pass: the same number of steps again with every launch bracketed by events
        # inside the library (pv_set_profiling). Those events are extra nodes of the attempt
        # graph and lengthen the step, so this pass only times the kernels.
        k.setProfiling(True)
        k.resetKernelStats()
        dt, _, pairs_profiled, _ = run_steps(dt, False)
        stats = k.kernelStats()
        k.setProfiling(False)
    total_ms = float(np.sum(step_ms))
    total_ms, pairs = combine_ranks(total_ms, pairs, f"cuda:{local}")
    value = pairs / (total_ms * 1e-3)

    # e2e: the same steps through the public API with host buffers -- every step uploads its
    # input state from pinned host memory and downloads the new state and the step result.
    e2e = measure_e2e(k, dt, max(10, args.steps // 4), local, SEED + rank)

    # roofline of the dominant kernel (the tiled periodic pair kernel), from its launch events
    # in the kernel pass: every timed velocity launch is one evaluation, its pairs over its time
    v_launch, v_timed, v_ms = stats["velocity"]
    per_launch_ms = v_ms / max(v_timed, 1)
    plan = k.statePlan()
    if plan["symmetric"]:
        flops_per_ordered_pair = FLOPS_PER_UNORDERED_PAIR_SYMMETRIC / 2.0
        kernel_name = "symmetric_kernel<PeriodicSym, 1>"
    else:
        flops_per_ordered_pair = FLOPS_PER_PAIR_PERIODIC
        kernel_name = "velocity_kernel<PeriodicPair>"
    achieved = flops_per_ordered_pair * pairs_profiled / (v_ms * 1e-3) / 1e12
    # measured FP64 FMA peak of this GPU (36.8 TFLOP/s at 1965 MHz on this pool's B200s when
    # the probe is skipped, e.g. under a profiler)
    peak = 36.83 if args.no_peak_probe else pv.probePeak("fp64", local) / 1e12

    result = None
    if rank == 0:
        result = {
            "metric": METRIC,
            "value": value,
            "unit": "pair-interactions/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64",
            "data": "synthetic (seeded uniform positions, balanced +-1 circulations)",
            "config": {"workload": WORKLOAD, "geometry": "periodic", "n_vortices": N,
                       "box_length": "2pi", "image_layers": LAYERS, "integrator": "dopri5",
                       "rtol": RTOL, "atol": ATOL, "dipole_threshold": DIPOLE_THRESHOLD,
                       "step": "one accepted DOPRI5 step + dipole scan",
                       "evaluations_per_rank": evals, "parallelism": f"replicas x{world}",
                       "l2": "256 MiB write between steps (outside the step timing)"},
            "e2e": e2e,
            "gpu_launches": int(launches),
            "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak,
                         "unit": "TFLOP/s", "frac": achieved / peak,
                         "traffic": TRAFFIC_BYTES_PER_LAUNCH,
                         "traffic_note": "DRAM bytes per launch (ncu); the algorithmic minimum "
                                         "is the 24N-byte source read, 98304 B",
                         "kernel": kernel_name,
                         "flops_per_pair": flops_per_ordered_pair,
                         "flops_executed_per_pair": (
                             FLOPS_EXECUTED_PER_UNORDERED_PAIR_SYMMETRIC / 2.0
                             if plan["symmetric"] else None),
                         "flops_note": "FP64 operations per ordered pair as the periodic series "
                                       "was first evaluated (FMA = 2), the implementation's own "
                                       "tally rather than a formula minimum, so frac reads as "
                                       "FP64-pipe work; kept fixed across kernel changes (the "
                                       "kernel now executes flops_executed_per_pair). "
                                       "Per ordered pair of the launched "
                                       "kernel (the symmetric form: 244 per unordered pair)",
                         "ms_per_launch": per_launch_ms, "launches": v_timed,
                         "timing": "CUDA events around each launch on the library stream, in a "
                                   "second pass of the same number of steps right after the "
                                   "timed one",
                         "peak_source": "measured FP64 FMA probe (pv_probe_peak) on this GPU"},
            "kernel_ms": {kk: vv[2] for kk, vv in stats.items()},
            "clocks": clocks.summary(),
        }
    return result, k


def measure_e2e(k, dt, steps, device, seed):
    """The step through the public API with HOST buffers: every step uploads the state from
    pinned host memory, takes the DOPRI5 step and the dipole events, and downloads the new state
    (positions and circulations, since events may change the population)."""
    import pointvortex_b200 as pv
    import torch
    s0 = k.downloadDeviceSystem()
    n = s0.size()
    host = torch.empty((3, n), dtype=torch.float64).pin_memory().numpy()
    host[0], host[1], host[2] = s0.x, s0.y, s0.circulation
    dipoles = dipole_manager(k, seed)
    evals = 0
    pairs = 0.0
    h2d = d2h = 0
    t0 = time.perf_counter()
    for _ in range(steps):
        st = pv.VortexSystem(host[0, :n], host[1, :n], host[2, :n])
        k.uploadDeviceState(st)
        before = k.evaluationCount
        r = k.deviceDopri5Step(dt, ATOL, RTOL, DTMIN, DTMAX)
        dipoles.process()
        e = k.evaluationCount - before
        out = k.downloadDeviceSystem()
        # x, y, circulation and the scaled circulations up; x, y, circulation down; the 256-byte
        # control block up once per attempt and down after each attempt and after the scan
        h2d += 32 * n + 256 * (1 + r.rejectedSteps)
        d2h += 24 * out.size() + 256 * (2 + r.rejectedSteps)
        pairs += e * n * (n - 1)
        n = out.size()
        host[0, :n], host[1, :n], host[2, :n] = out.x, out.y, out.circulation
        evals += e
        dt = r.suggestedTimeStep
    sec = time.perf_counter() - t0
    torch.cuda.synchronize(device)
    return {"value": pairs / sec, "unit": "pair-interactions/s",
            "h2d_bytes_per_step": h2d // steps, "d2h_bytes_per_step": d2h // steps,
            "steps": steps, "note": "upload + DOPRI5 step + dipole events + download per step; "
            "the upload invalidates FSAL, so each step makes 7 evaluations"}


def cpu_baseline(seconds: float = 10.0):
    """The reference's CPU/OpenMP periodic kernel on a bounded sample of targets of the same
    state, all host threads."""
    from oracle.pyoracle import Geometry, Oracle
    ics = load_ics()
    try:
        ref = Oracle("reference")
        kind = "reference"
    except FileNotFoundError:
        ref = Oracle("port")
        kind = "port"
    x, y, g = ics.periodic_box(N, SEED, LENGTH)
    geo = Geometry("periodic", box_length_x=LENGTH, box_length_y=LENGTH, image_layers=LAYERS)
    cores = ref.max_threads()
    ref.set_threads(cores)
    t0 = time.perf_counter()
    ref.evaluate_range(geo, x, y, g, 0, 16)
    t_probe = max(time.perf_counter() - t0, 1e-4)
    targets = int(min(N, max(16, 16 * seconds / t_probe)))
    t0 = time.perf_counter()
    ref.evaluate_range(geo, x, y, g, 0, targets)
    sec = time.perf_counter() - t0
    return {"value": targets * (N - 1) / sec, "unit": "pair-interactions/s", "cores": cores,
            "kind": kind, "sample": f"velocity of targets [0, {targets}) of the N={N} periodic "
            f"state against all {N} sources, {sec:.1f} s"}


# Wall-clock budget of the reference arm's timed steps: the arm stops timing after the step that
# crosses it (the metric is a rate, so fewer steps change its sample, not its meaning).
REFERENCE_TIMED_BUDGET_S = 150.0
REFERENCE_WARMUP_BUDGET_S = 60.0


def run_reference(args):
    """The reference's own CPU path of the same workload, all host threads: DOPRI5 steps of
    RungeKuttaIntegrator::dopri5Step (src/timestep.cpp:62-120, FSAL kept between steps) over
    PeriodicBoxKernel (src/compute.cpp:203-256), each followed by DipoleManager::process
    (src/dipole.cpp:42-127, removal at the workload's threshold) and the FSAL invalidation the
    driver makes after events (src/main.cpp:329-333). Unmodified reference code compiled into
    oracle/_ref (the port when it is absent); nothing of this repository's CUDA library is
    loaded."""
    rank, world, _ = rank_info()
    if rank != 0:
        return None
    from oracle.pyoracle import Geometry, Oracle
    ics = load_ics()
    try:
        ref = Oracle("reference")
        kind = "reference"
    except FileNotFoundError:
        ref = Oracle("port")
        kind = "port"
    x, y, g = ics.periodic_box(N, SEED, LENGTH)
    geo = Geometry("periodic", box_length_x=LENGTH, box_length_y=LENGTH, image_layers=LAYERS,
                   absolute_tolerance=ATOL, relative_tolerance=RTOL, minimum_time_step=DTMIN,
                   maximum_time_step=DTMAX, dipole_removal=True,
                   dipole_removal_distance=DIPOLE_THRESHOLD, random_seed=SEED)
    cores = ref.max_threads()
    ref.set_threads(cores)
    state = {"x": x, "y": y, "g": g, "dt": DT0, "fsal": False,
             "stepper": ref.stepper(geo, N), "n": N}

    def step():
        """One accepted DOPRI5 step + dipole events; returns the pair-interactions evaluated."""
        n = state["n"]
        nx, ny, res = state["stepper"].dopri5_step(state["x"], state["y"], state["g"], state["dt"])
        evals = (0 if state["fsal"] else 1) + 6 * (int(res[3]) + 1)
        state["fsal"] = True
        state["dt"] = float(res[1])
        if kind == "reference":
            events, nx, ny, ng = ref.dipole_process(geo, nx, ny, state["g"])
        else:
            events, ng = 0, state["g"]
        if events:
            state["stepper"] = ref.stepper(geo, nx.size)  # the driver invalidates FSAL
            state["fsal"] = False
            state["g"], state["n"] = ng, nx.size
        state["x"], state["y"] = nx, ny
        return evals * n * (n - 1)

    t0 = time.perf_counter()
    warm = 0
    for _ in range(max(args.warmup, 1)):  # the first step also takes the start-up rejections
        step()
        warm += 1
        if time.perf_counter() - t0 > REFERENCE_WARMUP_BUDGET_S:
            break
    pairs, timed = 0.0, 0
    t0 = time.perf_counter()
    for _ in range(args.steps):
        pairs += step()
        timed += 1
        if time.perf_counter() - t0 > REFERENCE_TIMED_BUDGET_S:
            break
    sec = time.perf_counter() - t0
    value = pairs / sec
    sample = (f"{timed} accepted DOPRI5 steps (of {args.steps} requested; {warm} warm-up) of the "
              f"N={N} periodic workload, each with the dipole events: the reference's "
              f"RungeKuttaIntegrator::dopri5Step over PeriodicBoxKernel and its DipoleManager, "
              f"N(N-1) pairs per evaluation")
    return {"metric": METRIC, "value": value, "unit": "pair-interactions/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3 / timed,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded uniform positions, balanced +-1 circulations)",
            "impl": "reference",
            "config": {"workload": WORKLOAD, "geometry": "periodic", "n_vortices": N,
                       "box_length": "2pi", "image_layers": LAYERS, "integrator": "dopri5",
                       "rtol": RTOL, "atol": ATOL, "dipole_threshold": DIPOLE_THRESHOLD,
                       "step": "one accepted DOPRI5 step + dipole scan"},
            "cpu_baseline": {"value": value, "unit": "pair-interactions/s", "cores": cores,
                             "kind": kind, "sample": sample, "steps_timed": timed},
            "e2e": {"value": value, "unit": "pair-interactions/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def run_kernel_case(spec: str, evals: int, precision: str = "fp64", ordered: bool = False) -> dict:
    """Velocity evaluations only (no stepping), for kernel timing and ncu captures:
    spec = "geometry:N" with geometry infinite | periodic | disk; precision fp64 | fp32c.
    ordered: evaluate host arrays (always the ordered-pair kernel) instead of the device state
    (the symmetric kernel where the plan uses it)."""
    import torch
    import pointvortex_b200 as pv
    from pointvortex_b200 import ics
    geo, n = spec.split(":")
    n = int(n)
    prec = 1 if precision == "fp32c" else 0
    if geo == "infinite":
        x, y, g = ics.infinite_plane(n, 1)
        k = pv.InfinitePlaneKernel(0.0, precision=prec)
        flops, flops_sym = FLOPS_PER_PAIR_PLANE, FLOPS_PER_UNORDERED_PAIR_PLANE_SYMMETRIC
    elif geo == "periodic":
        x, y, g = ics.periodic_box(n, 2, LENGTH)
        k = pv.PeriodicBoxKernel(LENGTH, LENGTH, LAYERS, precision=prec)
        flops, flops_sym = FLOPS_PER_PAIR_PERIODIC, FLOPS_PER_UNORDERED_PAIR_SYMMETRIC
    else:
        x, y, g = ics.disk(n, 3, 1.0)
        k = pv.DiskKernel(1.0, precision=prec)
        flops, flops_sym = 33, None
    k.uploadDeviceState(pv.VortexSystem(x, y, g))
    symmetric = k.statePlan()["symmetric"] and not ordered
    run = (lambda: k.evaluate(x, y, g)) if ordered else k.evaluateDeviceState
    for _ in range(2):
        run()
    k.setProfiling(True)
    k.resetKernelStats()
    for _ in range(evals):
        run()
    stats = k.kernelStats()
    st = stats["velocity"]
    ms = st[2] / max(st[1], 1)
    near_ms = stats["near"][2] / max(stats["near"][1], 1) if stats["near"][1] else 0.0
    pairs = n * (n - 1)
    work = (flops_sym * pairs / 2) if symmetric else flops * pairs
    torch.cuda.synchronize()
    return {"case": spec, "precision": precision, "kernel": "symmetric" if symmetric else "ordered",
            "evaluations": evals, "ms_per_evaluation": ms, "near_pass_ms": near_ms,
            "pairs_per_s": pairs / (ms * 1e-3),
            "formula_flops_per_pair": flops, "tflops": work / (ms * 1e-3) / 1e12,
            "ordered_equivalent_tflops": flops * pairs / (ms * 1e-3) / 1e12}


def run_reference_cuda(evals: int = 3, steps: int = 3) -> dict:
    """The reference's own CUDA backend (src/backend_cuda.cu, built for sm_100a into
    oracle/_ref/libpvref_cuda.so) on the same state: FP64, one thread per target, a host
    round trip after every evaluation. Runs in its own process."""
    import ctypes
    from oracle.pyoracle import REF_CUDA_LIB, _Params
    ics = load_ics()
    lib = ctypes.CDLL(REF_CUDA_LIB)
    D = ctypes.POINTER(ctypes.c_double)
    lib.pvref_stepper_create.restype = ctypes.c_void_p
    lib.pvref_stepper_create.argtypes = [ctypes.POINTER(_Params), ctypes.c_size_t]
    lib.pvref_device_upload.argtypes = [ctypes.c_void_p, D, D, D, ctypes.c_size_t]
    lib.pvref_device_evaluate.argtypes = [ctypes.c_void_p, D, D, ctypes.c_size_t]
    lib.pvref_device_dopri5_step.argtypes = [ctypes.c_void_p, ctypes.c_double, D]
    lib.pvref_last_error.restype = ctypes.c_char_p
    x, y, g = ics.periodic_box(N, SEED, LENGTH)
    par = _Params(1, 0.0, LENGTH, LENGTH, LAYERS, 1.0, ATOL, RTOL, DTMIN, DTMAX, 0, 0.01, 0, 1)
    h = lib.pvref_stepper_create(ctypes.byref(par), N)
    p = lambda a: a.ctypes.data_as(D)
    if lib.pvref_device_upload(h, p(x), p(y), p(g), N):
        return {"unavailable": lib.pvref_last_error().decode()}
    u, v = np.empty(N), np.empty(N)
    lib.pvref_device_evaluate(h, p(u), p(v), N)
    t0 = time.perf_counter()
    for _ in range(evals):
        lib.pvref_device_evaluate(h, p(u), p(v), N)
    t_eval = (time.perf_counter() - t0) / evals
    out = np.zeros(4)
    dt = DT0
    for _ in range(3):  # absorb the start-up rejections
        if lib.pvref_device_dopri5_step(h, dt, p(out)):
            return {"unavailable": lib.pvref_last_error().decode()}
        dt = out[1]
    t0 = time.perf_counter()
    for _ in range(steps):
        lib.pvref_device_dopri5_step(h, dt, p(out))
        dt = out[1]
    t_step = (time.perf_counter() - t0) / steps
    return {"impl": "reference CUDA backend (src/backend_cuda.cu, sm_100a)", "dtype": "f64",
            "ms_per_evaluation": t_eval * 1e3, "pairs_per_s": N * (N - 1) / t_eval,
            "ms_per_dopri5_step": t_step * 1e3,
            "note": "wall clock per call; the backend synchronises after every evaluation"}


def ensemble_specs(n_sims: int = 512, seed: int = 7) -> list:
    """The cfg-4 ensemble: N log-uniform in [64, 8192], geometry round-robin (infinite /
    periodic 2 pi / disk R = 1), one seed per simulation."""
    rng = np.random.default_rng(seed)
    geos = ("infinite", "periodic", "disk")
    specs = []
    for k in range(n_sims):
        n = int(np.exp(rng.uniform(np.log(64), np.log(8192))))
        n += n % 2
        specs.append((geos[k % 3], n, 1000 + k))
    return specs


def solve_batch(specs, budget: int, precision: str, device: int = 0):
    """Solves the given (geometry, N, seed) simulations in one batch: balanced +-1 circulations,
    DOPRI5 with rtol 1e-8 to t_end = 0.5, an accepted-step budget each. Returns (per-simulation
    (state, pairs), attempts, seconds from the first admission to the last result download)."""
    import torch
    from pointvortex_b200 import ics
    from pointvortex_b200.batch import Batch, geometry_params
    states = []
    for geo, n, sd in specs:
        if geo == "periodic":
            states.append(ics.periodic_box(n, sd, LENGTH))
        elif geo == "disk":
            states.append(ics.disk(n, sd, 1.0, 0.95, gaussian=False))
        else:
            states.append(ics.infinite_plane(n, sd))
    total = sum(n for _, n, _ in specs)
    b = Batch(total + 256 * (len(specs) + 1), max(len(specs), 1), device, max_steps=budget)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ids = [b.add(geometry_params(geo, precision=precision), *st, 0.5, dt=1e-3, atol=1e-10,
                 rtol=1e-8)
           for (geo, n, sd), st in zip(specs, states)]
    attempts = b.run() if ids else 0
    out = []
    for sid, (geo, n, sd) in zip(ids, specs):
        info = b.info(sid)
        b.result(sid)
        evals = 6 * (info.acceptedSteps + info.rejectedSteps) + 1
        out.append((info, float(evals) * n * (n - 1)))
    elapsed = time.perf_counter() - t0
    b.close()
    return out, attempts, elapsed


def run_ensemble(n_sims: int = 512, budget: int = 10, seed: int = 7,
                 precision: str = "fp64") -> dict:
    """Batched ensemble (cfg-4) on one GPU, each simulation with an accepted-step budget (the
    workloads are chaotic, so unbudgeted work per simulation is unbounded)."""
    specs = ensemble_specs(n_sims, seed)
    results, attempts, elapsed = solve_batch(specs, budget, precision)
    finished, reasons, per_thread = {}, {}, {}
    projected = {}
    for (info, _), (geo, n, _) in zip(results, specs):
        finished[info.state] = finished.get(info.state, 0) + 1
        kind = f"{geo}:{info.targetsPerThread}"  # 0: once-per-unordered-pair items
        per_thread[kind] = per_thread.get(kind, 0) + 1
        key = f"{geo}:{info.reason}"
        reasons[key] = reasons.get(key, 0) + 1
        if info.state == "budget" and info.time > 0:
            # accepted steps this simulation would need to reach t_end at its average step so far
            projected.setdefault(geo, []).append(info.acceptedSteps * 0.5 / info.time)
    pairs = sum(p for _, p in results)
    return {"simulations": n_sims, "vortices": sum(n for _, n, _ in specs), "step_budget": budget,
            "attempts": attempts, "seconds": elapsed, "budgeted_solves_per_s": n_sims / elapsed,
            "pair_interactions_per_s": pairs / elapsed, "states": finished,
            "stop_reasons": dict(sorted(reasons.items())),
            "targets_per_thread": dict(sorted(per_thread.items())),
            "projected_steps_to_t_end_median": {g: float(np.median(v)) for g, v in projected.items()},
            "dtype": "f64" if precision == "fp64" else "f32 compensated (f64 state and control)",
            "note": "one arena, lock-step DOPRI5 attempts, CUDA-graph replay per attempt; a "
                    "'budgeted solve' is a simulation that stopped (done, budget or failure), "
                    "not one that reached t_end"}


def run_ensemble_sharded(rank: int, world: int, device: int, n_sims: int = 512, budget: int = 10,
                         seed: int = 7) -> dict | None:
    """The same ensemble over `world` GPUs as replicas of the batch engine: each rank solves its
    share of the simulations (cost-balanced partition), only the results go to rank 0. The time
    is the slowest rank's."""
    import torch.distributed as dist
    from pointvortex_b200.shard import run_sharded, simulation_cost, torch_gather
    specs = ensemble_specs(n_sims, seed)
    timing = {}

    def run_local(mine):
        # never raises: every rank must reach the gathers
        try:
            results, _, elapsed = solve_batch([s for _, s in mine], budget, "fp64", device)
        except Exception as exc:
            timing["error"] = str(exc)[:200]
            return []
        timing["seconds"] = elapsed
        return [(i, (info.reason, pairs)) for (i, _), (info, pairs) in zip(mine, results)]

    dist.barrier()
    merged = run_sharded(specs, lambda s: simulation_cost(s[0], s[1]), run_local, rank, world,
                         torch_gather)
    seconds = max(torch_gather(timing.get("seconds", 0.0)))
    errors = [e for e in torch_gather(timing.get("error")) if e]
    if rank != 0:
        return None
    if errors or any(m is None for m in merged):
        return {"error": (errors or ["a rank returned no results"])[0]}
    pairs = sum(p for _, p in merged)
    reasons = {}
    for reason, _ in merged:
        reasons[reason] = reasons.get(reason, 0) + 1
    return {"simulations": n_sims, "ranks": world, "seconds": seconds,
            "budgeted_solves_per_s": n_sims / seconds, "pair_interactions_per_s": pairs / seconds,
            "stop_reasons": reasons,
            "note": "replicas: one batch engine per GPU, cost-balanced partition, results "
                    "gathered once"}


# The serving sweep: request counts per arrival rate (20,000 per rate, as the configuration states,
# would take about 8 minutes of GPU time per rate and arm at the ~40 solves/s these budgets allow;
# each rate runs this many requests, the same for the server and the comparison loop).
SERVING_STREAMS = ((10.0, 100), (30.0, 200), (100.0, 300), (300.0, 300), (1000.0, 300))


def run_serving(budget: int = 10, streams=SERVING_STREAMS) -> dict:
    """Continuous-batching server on Poisson request streams (geometry uniform, N log-uniform in
    [32, 32768], t_end U[0.1, 1], rtol in {1e-6, 1e-9}, accepted-step budget per request), and the
    one-request-at-a-time FIFO loop on the same stream at every rate."""
    from pointvortex_b200.serve import Server, one_at_a_time, poisson_stream
    out = {"step_budget": budget, "requests_per_rate": {str(r): c for r, c in streams},
           "note": "the configuration's 20000 requests per rate are cut to the counts given, the "
                   "same for both arms, to keep the sweep within minutes",
           "server": [], "one_request_per_launch_fp64": []}
    for rate, count in streams:
        reqs = poisson_stream(count, rate, seed=int(rate), max_steps=budget)
        # split_context: cheap requests share batched launches (16 attempts per call), expensive
        # ones run one at a time on single-simulation contexts (each fills the GPU alone and
        # gets the fastest kernels, the periodic box once per unordered pair), the two lanes on
        # their own host threads and streams; waiting requests are admitted shortest work first;
        # a cheap request that finds its lane idle is solved at once on a context. Measured
        # against policy "split" (the expensive requests batched too): higher throughput and
        # lower p50 and p99 at every rate.
        server = Server(capacity_vortices=4_000_000, max_slots=1024, attempts_per_tick=2,
                        policy="split_context", order="sjf", solo_max_steps=64)
        summary = server.serve(reqs)
        server.close()
        summary["rate_per_s"] = rate
        out["server"].append(summary)
        base = one_at_a_time(poisson_stream(count, rate, seed=int(rate), max_steps=budget))
        base["rate_per_s"] = rate
        out["one_request_per_launch_fp64"].append(base)
    return out


def reference_rk4_drift(x, y, g, steps: int = 100, dt: float = 1e-3) -> dict:
    """The invariants' drift of the reference's own CPU run of the same RK4 case
    (RungeKuttaIntegrator::rk4Step, src/timestep.cpp:31-61; computeInvariants,
    src/compute.cpp:134-163), printed beside the GPU's: H and L are not conserved by RK4 at this
    step, so their drift is compared in size, not value."""
    from oracle.pyoracle import Geometry, Oracle
    try:
        ref = Oracle("reference")
    except FileNotFoundError:
        return {"unavailable": "oracle/_ref was not built"}
    ref.set_threads(ref.max_threads())
    geo = Geometry("infinite")
    inv0 = ref.invariants(geo, x, y, g)
    st = ref.stepper(geo, x.size)
    cx, cy = x.copy(), y.copy()
    for _ in range(steps):
        cx, cy = st.rk4_step(cx, cy, g, dt)
    d = ref.invariants(geo, cx, cy, g) - inv0
    return {"circulation": float(d[0]), "linear_impulse_x": float(d[1]),
            "linear_impulse_y": float(d[2]), "angular_impulse": float(d[3]),
            "hamiltonian": float(d[4]), "kind": "reference CPU (oracle/_ref)"}


def run_other_configs() -> dict:
    """The other single-simulation configurations, timed on the device (CUDA events of the
    library's launches):
    * infinite plane N = 1024, RK4 dt = 1e-3, 100 steps (pv_rk4_advance): pair-interactions/s
      and the invariants' drift over the run;
    * disk N = 16384 (Gaussian circulations), plain FP64 and FP32-compensated evaluations:
      pair-interactions/s of each and the FP32C velocity's error against the FP64 one. Its RK4
      run at dt = 5e-4 leaves the disk at step 1 in the reference, and here alike (reported)."""
    import torch
    import pointvortex_b200 as pv
    from pointvortex_b200 import ics
    out = {}
    x, y, g = ics.workload_state("infinite_rk4_n1024")
    k = pv.InfinitePlaneKernel(0.0)
    k.uploadDeviceState(pv.VortexSystem(x, y, g))
    inv0 = k.stateInvariants()
    k.rk4Advance(1e-3, 5)
    k.uploadDeviceState(pv.VortexSystem(x, y, g))
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stream = torch.cuda.ExternalStream(k.cudaStream())
    start.record(stream)
    k.rk4Advance(1e-3, 100)
    stop.record(stream)
    torch.cuda.synchronize()
    ms = start.elapsed_time(stop)
    inv1 = k.stateInvariants()
    out["infinite_rk4_n1024"] = {
        "steps": 100, "ms": ms, "ms_per_step": ms / 100,
        "pair_interactions_per_s": 400 * 1024 * 1023 / (ms * 1e-3),
        "drift": {"circulation": inv1.circulation - inv0.circulation,
                  "linear_impulse_x": inv1.linearImpulseX - inv0.linearImpulseX,
                  "linear_impulse_y": inv1.linearImpulseY - inv0.linearImpulseY,
                  "angular_impulse": inv1.angularImpulse - inv0.angularImpulse,
                  "hamiltonian": inv1.hamiltonian - inv0.hamiltonian},
        "note": "the 100 steps are one cooperative launch (pv_rk4_advance, N <= 2048)"}
    out["infinite_rk4_n1024"]["reference_drift"] = reference_rk4_drift(x, y, g)
    x, y, g = ics.workload_state("disk_rk4_n16384")
    forms = {}
    vel = {}
    for name, prec in (("fp64", 0), ("fp32c", 1)):
        kd = pv.DiskKernel(1.0, precision=prec)
        kd.uploadDeviceState(pv.VortexSystem(x, y, g))
        kd.evaluateDeviceState()
        kd.setProfiling(True)
        kd.resetKernelStats()
        for _ in range(10):
            vel[name] = kd.evaluateDeviceState()
        st = kd.kernelStats()
        # one evaluation: the velocity launch, the FP32C form's FP64 near-field pass, the reduction
        per = (st["velocity"][2] + st["near"][2] + st["stage"][2]) / max(st["stage"][1], 1)
        forms[name] = {"ms_per_evaluation": per, "pair_interactions_per_s": 16384 * 16383 / (per * 1e-3),
                       "velocity_kernel_ms": st["velocity"][2] / max(st["velocity"][1], 1),
                       "near_pass_ms": st["near"][2] / max(st["near"][1], 1) if st["near"][1] else 0.0,
                       "reduction_ms": st["stage"][2] / max(st["stage"][1], 1)}
        try:
            kd.deviceRk4Step(5e-4)
            forms[name]["rk4_step_1"] = "ok"
        except (RuntimeError, ValueError) as exc:
            forms[name]["rk4_step_1"] = str(exc)
    a, b = vel["fp64"], vel["fp32c"]
    mag = np.hypot(a.x, a.y)
    scale = np.maximum(mag, np.sqrt(np.mean(mag * mag)))
    err = np.hypot(b.x - a.x, b.y - a.y) / scale
    forms["fp32c_vs_fp64_error"] = {"max": float(err.max()), "rms": float(np.sqrt(np.mean(err ** 2)))}
    forms["speedup"] = forms["fp32c"]["pair_interactions_per_s"] / forms["fp64"]["pair_interactions_per_s"]
    out["disk_n16384"] = forms
    return out


def run_fp32c_curve(reps: int = 10) -> dict:
    """Error and speed of the FP32-compensated form against its near-field radius, on the periodic
    workload state (N = 4096, symmetric kernel), a periodic state of N = 16384, and the disk
    workload state (N = 16384, Gaussian circulations, ordered kernel): per radius (in units of the mean spacing; 0 = no near field) the
    per-vortex error against the FP64 kernel (itself within 1e-12 of the oracle) and the time per
    evaluation, next to the FP64 kernel's."""
    import torch
    import pointvortex_b200 as pv
    from pointvortex_b200 import ics
    out = {}
    cases = [("periodic_n4096", lambda p: pv.PeriodicBoxKernel(LENGTH, LENGTH, LAYERS, precision=p),
              ics.workload_state("periodic_dopri5_n4096"), LENGTH / np.sqrt(4096)),
             ("periodic_n16384", lambda p: pv.PeriodicBoxKernel(LENGTH, LENGTH, LAYERS, precision=p),
              ics.periodic_box(16384, 20240104, LENGTH), LENGTH / np.sqrt(16384)),
             ("disk_n16384", lambda p: pv.DiskKernel(1.0, precision=p),
              ics.workload_state("disk_rk4_n16384"), np.sqrt(np.pi / 16384))]

    def timed(k):
        k.evaluateDeviceState()
        k.setProfiling(True)
        k.resetKernelStats()
        for _ in range(reps):
            f = k.evaluateDeviceState()
        st = k.kernelStats()
        k.setProfiling(False)
        ms = (st["velocity"][2] + st["near"][2] + st["stage"][2]) / max(st["stage"][1], 1)
        return f, ms

    for name, make, (x, y, g), spacing in cases:
        k64 = make(0)
        k64.uploadDeviceState(pv.VortexSystem(x, y, g))
        ref, ms64 = timed(k64)
        mag = np.hypot(ref.x, ref.y)
        scale = np.maximum(mag, np.sqrt(np.mean(mag * mag)))
        rows = []
        k32 = make(1)
        k32.uploadDeviceState(pv.VortexSystem(x, y, g))
        for units in (0.0, 0.5, 1.0, 2.0, 4.0, 8.0):
            k32.setNearField(units * spacing)
            f, ms = timed(k32)
            err = np.hypot(f.x - ref.x, f.y - ref.y) / scale
            rows.append({"radius_spacings": units, "radius": units * spacing,
                         "max": float(err.max()), "rms": float(np.sqrt(np.mean(err ** 2))),
                         "ms_per_evaluation": ms, "speedup_vs_fp64": ms64 / ms})
        k32.setNearField(-1.0)
        out[name] = {"fp64_ms_per_evaluation": ms64, "default_radius": k32.nearField,
                     "curve": rows, "note": "evaluation = velocity launch + FP64 near-field pass + "
                                            "reduction stage (CUDA events around each launch)"}
        k32.close()
        k64.close()
    torch.cuda.synchronize()
    return out


def run_output(reps: int = 10) -> dict:
    """The reference's text output at GPU rates: one trajectory frame (TrajectoryWriter::write,
    velocity evaluated on the device) and one checkpoint vortex block of the N = 16384 disk
    workload state, formatted on the GPU, copied to the host and written to a file; wall clock
    per frame, plus the formatting kernels' own time from their launch events."""
    import tempfile
    import pointvortex_b200 as pv
    from pointvortex_b200 import ics
    x, y, g = ics.workload_state("disk_rk4_n16384")
    k = pv.DiskKernel(1.0)
    k.uploadDeviceState(pv.VortexSystem(x, y, g))
    out = {"workload": "disk_n16384", "rows": int(x.size)}
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "trajectory.csv")
        for name, call in (("trajectory_frame", lambda: k.formatTrajectory(0.1, 1)),
                           ("checkpoint_block", k.formatCheckpointVortices)):
            with open(path, "wb") as f:
                for _ in range(3):
                    f.write(call())
                k.setProfiling(True)
                k.resetKernelStats()
                t0 = time.perf_counter()
                for _ in range(reps):
                    text = call()
                    f.write(text)
                    f.flush()
                sec = (time.perf_counter() - t0) / reps
                stats = k.kernelStats()
                k.setProfiling(False)
            launches, timed, ms = stats["output"]
            kernel_ms = ms / max(timed, 1)
            out[name] = {"ms_per_frame": sec * 1e3, "bytes": len(text),
                         "formatting_kernels_ms": kernel_ms,
                         "formatted_GB_per_s": len(text) / (kernel_ms * 1e-3) / 1e9}
        vel = k.evaluateDeviceState()
    out["inputs"] = (x, y, g, vel.x, vel.y)
    return out


def cpu_baseline_output(inputs, reps: int = 3) -> dict:
    """The reference's own TrajectoryWriter (src/print.cpp, compiled into oracle/_ref) writing
    the same frame on the host: the CPU baseline of the output row."""
    import tempfile
    from oracle.pyoracle import Oracle
    try:
        ref = Oracle("reference")
    except FileNotFoundError as exc:
        return {"unavailable": str(exc)[:200]}
    x, y, g, u, v = inputs
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "trajectory.csv")
        ref.write_trajectory(path, 0.1, 1, x, y, g, u, v)
        t0 = time.perf_counter()
        for _ in range(reps):
            ref.write_trajectory(path, 0.1, 1, x, y, g, u, v)
        sec = (time.perf_counter() - t0) / reps
    return {"ms_per_frame": sec * 1e3, "kind": "reference", "cores": 1,
            "sample": f"TrajectoryWriter::write of the same {x.size}-row frame into a new file"}


def summarize_launches(path: str) -> str:
    """Per-kernel launches, total time and share of an ncu launch list
    (`ncu --metrics gpu__time_duration.sum --csv --log-file <path> ...`), as a Markdown table."""
    import csv
    import re
    from collections import defaultdict
    with open(path) as f:
        lines = [ln for ln in f if ln.startswith('"')]
    total, count = defaultdict(float), defaultdict(int)
    for r in csv.DictReader(lines):
        if r.get("Metric Name") != "gpu__time_duration.sum":
            continue
        k = re.sub(r"\(.*", "", r["Kernel Name"]).replace("pvb::", "")
        k = k.replace("(anonymous namespace)::", "")[:70]
        scale = {"nsecond": 1e-3, "usecond": 1.0, "msecond": 1e3, "second": 1e6}.get(
            r.get("Metric Unit", "nsecond"), 1e-3)
        total[k] += float(r["Metric Value"].replace(",", "")) * scale
        count[k] += 1
    grand = sum(total.values()) or 1.0
    out = ["| kernel | launches | total (us) | share |", "|---|---|---|---|"]
    for k in sorted(total, key=total.get, reverse=True):
        out.append(f"| `{k}` | {count[k]} | {total[k]:.1f} | {100 * total[k] / grand:.1f} % |")
    out.append(f"| all | {sum(count.values())} | {grand:.1f} | 100 % |")
    return "\n".join(out)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the ensemble and serving sections")
    ap.add_argument("--kernel-case", default=None,
                    help="geometry:N -- time velocity evaluations only (kernel timing / ncu)")
    ap.add_argument("--evals", type=int, default=10)
    ap.add_argument("--precision", choices=["fp64", "fp32c"], default="fp64",
                    help="precision form of --kernel-case")
    ap.add_argument("--ordered", action="store_true",
                    help="--kernel-case on host arrays: the ordered-pair kernel")
    ap.add_argument("--reference-cuda", action="store_true",
                    help="time the reference's own CUDA backend on the workload (own process)")
    ap.add_argument("--summarize-launches", default=None, metavar="CSV",
                    help="print the per-kernel summary of an ncu launch list and exit")
    ap.add_argument("--no-peak-probe", action="store_true",
                    help="report the roofline against the last measured FP64 peak")
    ap.add_argument("--fp32c-curve", action="store_true",
                    help="print the FP32C error and speed against the near-field radius and exit")
    ap.add_argument("--section", choices=["serving", "ensemble", "other"], default=None,
                    help="run one of the extra sections alone, print its JSON and exit")
    args = ap.parse_args(argv)
    rank, world, _ = rank_info()
    if args.summarize_launches:
        print(summarize_launches(args.summarize_launches))
        return 0
    if args.reference_cuda:
        print(json.dumps(run_reference_cuda()), flush=True)
        return 0
    if args.section:
        run = {"serving": run_serving, "other": run_other_configs,
               "ensemble": lambda: {"fp64": run_ensemble(),
                                    "fp32c": run_ensemble(precision="fp32c")}}[args.section]
        print(json.dumps(run()), flush=True)
        return 0
    if args.fp32c_curve:
        print(json.dumps(run_fp32c_curve()), flush=True)
        return 0
    if args.kernel_case:
        print(json.dumps(run_kernel_case(args.kernel_case, args.evals, args.precision,
                                         args.ordered)), flush=True)
        return 0
    if args.impl == "reference":
        out = run_reference(args)
        if out is not None:
            print(json.dumps(out), flush=True)
        return 0
    result, k = run_ours(args)
    if world > 1 and not args.no_extras:
        try:  # every rank takes part (collectives in the same order everywhere)
            sharded = run_ensemble_sharded(rank, world, int(os.environ.get("LOCAL_RANK", "0")))
        except Exception as exc:
            sharded = {"error": str(exc)[:200]}
        if rank == 0:
            result["ensemble_sharded"] = sharded
    if rank == 0 and world == 1 and not args.no_extras:
        try:
            result["ensemble"] = run_ensemble()
            result["ensemble_fp32c"] = run_ensemble(precision="fp32c")
        except Exception as exc:
            result["ensemble"] = {"error": str(exc)[:200]}
        try:
            result["serving"] = run_serving()
        except Exception as exc:
            result["serving"] = {"error": str(exc)[:200]}
        try:
            result["other_configs"] = run_other_configs()
        except Exception as exc:
            result["other_configs"] = {"error": str(exc)[:200]}
        try:
            result["fp32c_near_field"] = run_fp32c_curve()
        except Exception as exc:
            result["fp32c_near_field"] = {"error": str(exc)[:200]}
        try:
            out = run_output()
            inputs = out.pop("inputs")
            if not args.no_cpu_baseline:
                out["reference_cpu"] = cpu_baseline_output(inputs)
            result["output"] = out
        except Exception as exc:
            result["output"] = {"error": str(exc)[:200]}
    if rank == 0:
        if not args.no_cpu_baseline and world == 1:
            result["cpu_baseline"] = cpu_baseline()
            try:
                rc = subprocess.run([sys.executable, os.path.abspath(__file__), "--reference-cuda"],
                                    capture_output=True, text=True, timeout=300)
                ref_gpu = json.loads(rc.stdout.strip().splitlines()[-1])
                if "ms_per_dopri5_step" in ref_gpu:
                    ref_gpu["speedup_per_dopri5_step"] = (ref_gpu["ms_per_dopri5_step"]
                                                          / result["ms_per_step"])
                result["reference_cuda_fp64"] = ref_gpu
            except Exception as exc:  # reported, never fatal to the benchmark line
                result["reference_cuda_fp64"] = {"unavailable": str(exc)[:200]}
        print(json.dumps(result), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
