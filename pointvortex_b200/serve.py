"""Continuous-batching solve server over the batched ensemble engine.

A request is one solve: (geometry, N, seed, t_end, tolerance). The server keeps every admitted
state resident in one device arena. New requests are admitted whenever a slot and arena room (the
HBM budget) are free, including while others are mid-flight, and they join the next batched
DOPRI5 attempt. Finished solves are retired, their final states downloaded and handed to a
callback (streamed), and their room freed. Latency is measured from arrival to retirement.

`one_at_a_time()` is the comparison loop: the same requests, FIFO, each solved alone with the
single-simulation context API (one simulation per launch, plain FP64).
"""
from __future__ import annotations

import heapq
import time
from dataclasses import dataclass, field
from typing import Callable, Optional

import numpy as np

from . import ics
from .batch import Batch, CapacityError, geometry_params


@dataclass
class Request:
    rid: int
    geometry: str
    n: int
    seed: int
    t_end: float
    rtol: float
    atol: float = 1e-12
    dt: float = 1e-3
    max_steps: int = 0
    arrival: float = 0.0          # seconds after the start of the stream

    def state(self):
        if self.geometry == "periodic":
            return ics.periodic_box(self.n + self.n % 2, self.seed)
        if self.geometry == "disk":
            return ics.disk(self.n, self.seed, 1.0, 0.95, gaussian=False)
        return ics.infinite_plane(self.n, self.seed)


@dataclass
class Completion:
    rid: int
    state: str                    # done | budget | failed
    latency: float                # seconds, arrival -> retirement
    accepted_steps: int
    time: float
    x: Optional[np.ndarray] = None
    y: Optional[np.ndarray] = None


def poisson_stream(n_requests: int, rate: float, seed: int, n_min: int = 32, n_max: int = 32768,
                   t_end_range=(0.1, 1.0), rtols=(1e-6, 1e-9), max_steps: int = 0) -> list[Request]:
    """Requests with exponential inter-arrival times (rate per second): geometry uniform over the
    three, N log-uniform in [n_min, n_max], t_end uniform, rtol drawn from `rtols`."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    geos = ("infinite", "periodic", "disk")
    for k in range(n_requests):
        t += rng.exponential(1.0 / rate)
        n = int(np.exp(rng.uniform(np.log(n_min), np.log(n_max))))
        geo = geos[int(rng.integers(3))]
        if geo == "periodic":
            n += n % 2
        out.append(Request(k, geo, max(n, 2), int(rng.integers(1 << 31)),
                           float(rng.uniform(*t_end_range)), float(rtols[int(rng.integers(len(rtols)))]),
                           max_steps=max_steps, arrival=t))
    return out


class Server:
    def __init__(self, capacity_vortices: int, max_slots: int, attempts_per_tick: int = 4,
                 device: int = 0, keep_states: bool = False):
        self.batch = Batch(capacity_vortices, max_slots, device)
        self.attempts_per_tick = attempts_per_tick
        self.keep_states = keep_states
        self.queue: list = []          # (arrival, rid, request) min-heap, FIFO by arrival
        self.running: dict[int, tuple] = {}
        self.completions: list[Completion] = []

    def submit(self, req: Request) -> None:
        heapq.heappush(self.queue, (req.arrival, req.rid, req))

    def _admit(self, now: float) -> int:
        admitted = 0
        while self.queue and self.queue[0][0] <= now:
            _, _, req = self.queue[0]
            x, y, g = req.state()
            try:
                sid = self.batch.add(geometry_params(req.geometry), x, y, g, req.t_end, dt=req.dt,
                                     atol=req.atol, rtol=req.rtol, max_steps=req.max_steps)
            except CapacityError:
                break                   # wait for room: head-of-line, arrival order kept
            heapq.heappop(self.queue)
            self.running[sid] = (req, now)
            admitted += 1
        return admitted

    def _retire(self, now: float, on_complete) -> int:
        done = 0
        for sid in list(self.running):
            info = self.batch.info(sid)
            if info.state == "running":
                continue
            req, _ = self.running.pop(sid)
            x = y = None
            if self.keep_states or on_complete is not None:
                x, y = self.batch.result(sid)
            self.batch.release(sid)
            c = Completion(req.rid, info.state, now - req.arrival, info.acceptedSteps, info.time,
                           x if self.keep_states else None, y if self.keep_states else None)
            self.completions.append(c)
            if on_complete is not None:
                on_complete(c, x, y)
            done += 1
        return done

    def serve(self, requests: list[Request], on_complete: Optional[Callable] = None,
              clock=time.perf_counter) -> dict:
        """Runs the stream in real time: a request becomes visible at its arrival time."""
        for r in requests:
            self.submit(r)
        start = clock()
        total = len(requests)
        while len(self.completions) < total:
            now = clock() - start
            self._admit(now)
            if not self.running:
                if self.queue:
                    wait = self.queue[0][0] - (clock() - start)
                    if wait > 0:
                        time.sleep(min(wait, 0.01))
                continue
            self.batch.advance(self.attempts_per_tick)
            self._retire(clock() - start, on_complete)
        elapsed = clock() - start
        return summarize(self.completions, elapsed)

    def close(self):
        self.batch.close()


def summarize(completions: list[Completion], elapsed: float) -> dict:
    lat = np.array([c.latency for c in completions]) if completions else np.zeros(1)
    states = {}
    for c in completions:
        states[c.state] = states.get(c.state, 0) + 1
    return {"requests": len(completions), "elapsed_s": elapsed,
            "solves_per_s": len(completions) / elapsed if elapsed > 0 else 0.0,
            "p50_latency_s": float(np.percentile(lat, 50)),
            "p99_latency_s": float(np.percentile(lat, 99)), "states": states}


def one_at_a_time(requests: list[Request], device: int = 0, clock=time.perf_counter) -> dict:
    """FIFO baseline: each request solved alone through the single-simulation context API
    (pv_upload_state + pv_dopri5_step per step), in arrival order."""
    from .kernel import DiskKernel, InfinitePlaneKernel, PeriodicBoxKernel, VortexSystem
    kernels = {"infinite": InfinitePlaneKernel(0.0, device=device),
               "periodic": PeriodicBoxKernel(2 * np.pi, 2 * np.pi, 8, device=device),
               "disk": DiskKernel(1.0, device=device)}
    out = []
    start = clock()
    for req in sorted(requests, key=lambda r: r.arrival):
        now = clock() - start
        if req.arrival > now:
            time.sleep(req.arrival - now)
        k = kernels[req.geometry]
        x, y, g = req.state()
        k.uploadDeviceState(VortexSystem(x, y, g))
        t, dt, steps, state = 0.0, min(max(req.dt, 1e-12), 0.1), 0, "done"
        try:
            while t < req.t_end:
                if req.max_steps and steps >= req.max_steps:
                    state = "budget"
                    break
                r = k.deviceDopri5Step(min(dt, req.t_end - t), req.atol, req.rtol, 1e-12, 0.1)
                t += r.acceptedTimeStep
                dt = r.suggestedTimeStep
                steps += 1
                if t + 16 * np.finfo(float).eps * abs(t) >= req.t_end:
                    t = req.t_end
        except (RuntimeError, ValueError):
            state = "failed"
        out.append(Completion(req.rid, state, clock() - start - req.arrival, steps, t))
    return summarize(out, clock() - start)
