"""Continuous-batching solve server over the batched ensemble engine.

A request is one solve: (geometry, N, seed, t_end, tolerance). The server keeps every admitted
state resident in a device arena. New requests are admitted whenever a slot and arena room (the
HBM budget) are free, including while others are mid-flight, and they join the next batched
DOPRI5 attempt. Finished solves are retired, their final states downloaded and handed to a
callback (streamed), and their room freed. Latency is measured from arrival to retirement.

In a lock-step attempt every simulation advances once, so a batch moves at the pace of its most
expensive member. With policy "split" the server also admits by estimated work: cheap requests
(one evaluation at most `split_work` plane-pair units) go to their own batch, which takes several
attempts for each attempt of the batch holding the expensive ones. Both are batches -- the
expensive requests share their launches too -- each driven by its own host thread on its own CUDA
stream, so their kernels overlap on the GPU. Within a lane, waiting requests are admitted
shortest estimated work first (order="sjf") or in arrival order (order="fifo").

`one_at_a_time()` is the comparison loop: the same requests, FIFO, each solved alone with the
single-simulation context API (one simulation per launch, plain FP64).
"""
from __future__ import annotations

import heapq
import threading
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
    pairs: float = 0.0            # pair interactions evaluated for this request
    engine: str = "batch"         # batch: in a batched launch; context: alone on a context


# Relative cost of one ordered pair by geometry, from the measured FP64 pair rates of the
# single-simulation kernels (plane 1.5e12, disk 5.3e11, periodic 9.6e10 pairs/s).
PAIR_COST = {"infinite": 1.0, "disk": 2.9, "periodic": 15.8}


def work(req: "Request") -> float:
    """Estimated cost of one velocity evaluation of the request, in plane-pair units."""
    return PAIR_COST[req.geometry] * float(req.n) * float(req.n)


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


class _Lane:
    """One batch with its own queue of arrived requests. solo_max_steps > 0: a request that finds
    the lane idle and alone in its queue, with a step budget of at most solo_max_steps, is solved
    at once on the lane's own single-simulation contexts instead (a batch of one pays the batched
    attempt's fixed launches; a context runs the attempt as one graph)."""

    def __init__(self, capacity_vortices: int, max_slots: int, device: int, attempts: int,
                 solo_max_steps: int = 0):
        self.batch = Batch(capacity_vortices, max_slots, device)
        self.attempts = attempts
        self.ready: list = []            # (arrival, rid, request), in admission order
        self.running: dict[int, tuple] = {}
        self.solo_max_steps = solo_max_steps
        self.kernels = _contexts(device) if solo_max_steps > 0 else None

    def take_solo(self):
        """The request to solve alone now, removed from the queue, or None."""
        if (self.kernels is None or self.running or len(self.ready) != 1 or
                not 0 < self.ready[0][2].max_steps <= self.solo_max_steps):
            return None
        return self.ready.pop(0)[2]

    def run_solo(self, server: "Server", req: "Request", clock, start: float, want_states: bool):
        """(completion, x, y): the request solved alone; x, y the final positions if wanted."""
        solver = _Solver(self.kernels, req)
        while not solver.step():
            pass
        x = y = None
        if server.keep_states or want_states:
            x, y = solver.positions()
        c = Completion(req.rid, solver.state, clock() - start - req.arrival, solver.steps,
                       solver.t, x if server.keep_states else None,
                       y if server.keep_states else None, solver.pairs(), engine="context")
        return c, x, y

    def admit(self, server: "Server", now: float) -> int:
        return server._admit_lane(self, now)

    def advance(self) -> None:
        self.batch.advance(self.attempts)

    def retire(self, server: "Server", now: float, on_complete) -> int:
        return server._retire(self, now, on_complete)

    def close(self) -> None:
        self.batch.close()
        for k in (self.kernels or {}).values():
            k.close()


class _Solver:
    """The reference driver's DOPRI5 loop (src/main.cpp:310-343, without output events) for one
    request on a single-simulation context: its own step size, end-time landing and budget."""

    def __init__(self, kernels: dict, req: Request):
        from .kernel import VortexSystem
        self.req = req
        self.k = kernels[req.geometry]
        x, y, g = req.state()
        self.k.uploadDeviceState(VortexSystem(x, y, g))
        self.t, self.dt, self.steps = 0.0, min(max(req.dt, 1e-12), 0.1), 0
        self.state: Optional[str] = None
        self.evals0 = self.k.evaluationCount

    def step(self) -> bool:
        """One accepted step; True once the solve has ended (done, budget or failed)."""
        req = self.req
        if self.t >= req.t_end:
            self.state = "done"
            return True
        if req.max_steps and self.steps >= req.max_steps:
            self.state = "budget"
            return True
        try:
            r = self.k.deviceDopri5Step(min(self.dt, req.t_end - self.t), req.atol, req.rtol,
                                        1e-12, 0.1)
        except (RuntimeError, ValueError):
            self.state = "failed"
            return True
        self.t += r.acceptedTimeStep
        self.dt = r.suggestedTimeStep
        self.steps += 1
        if self.t + 16 * np.finfo(float).eps * abs(self.t) >= req.t_end:
            self.t = req.t_end
        return False

    def pairs(self) -> float:
        return float(self.k.evaluationCount - self.evals0) * self.req.n * (self.req.n - 1)

    def positions(self):
        from .kernel import VortexSystem
        n = self.k.stateSize()
        st = VortexSystem(np.zeros(n), np.zeros(n), np.zeros(n))
        self.k.downloadDeviceState(st)
        return st.x, st.y


def _contexts(device: int) -> dict:
    from .kernel import DiskKernel, InfinitePlaneKernel, PeriodicBoxKernel
    return {"infinite": InfinitePlaneKernel(0.0, device=device),
            "periodic": PeriodicBoxKernel(2 * np.pi, 2 * np.pi, 8, device=device),
            "disk": DiskKernel(1.0, device=device)}


class _ContextLane:
    """Expensive requests, one at a time, each on a single-simulation context: one such request
    fills the GPU by itself, and the context runs the fastest kernels for it (the periodic box
    once per unordered pair)."""

    def __init__(self, device: int, steps_per_call: int):
        self.kernels = _contexts(device)
        self.steps_per_call = steps_per_call
        self.ready: list = []
        self.current: Optional[tuple] = None   # (solver, admitted at)
        self.running: dict = {}

    def admit(self, server: "Server", now: float) -> int:
        if self.current is not None or not self.ready:
            return 0
        _, _, req = self.ready.pop(0)
        self.current = (_Solver(self.kernels, req), now)
        self.running = {req.rid: self.current}
        return 1

    def advance(self) -> None:
        solver = self.current[0]
        for _ in range(self.steps_per_call):
            if solver.step():
                break

    def retire(self, server: "Server", now: float, on_complete) -> int:
        solver = self.current[0]
        if solver.state is None:
            return 0
        req = solver.req
        x = y = None
        if server.keep_states or on_complete is not None:
            x, y = solver.positions()
        c = Completion(req.rid, solver.state, now - req.arrival, solver.steps, solver.t,
                       x if server.keep_states else None, y if server.keep_states else None,
                       solver.pairs(), engine="context")
        server.completions.append(c)
        if on_complete is not None:
            on_complete(c, x, y)
        self.current = None
        self.running = {}
        return 1

    def close(self) -> None:
        for k in self.kernels.values():
            k.close()


class Server:
    """Continuous batching. policy "fifo": one batch. policy "split" (admission by estimated
    work): requests whose evaluation costs at most `split_work` plane-pair units go to a cheap
    batch, which takes `small_attempts` attempts per call; the expensive ones go to a second
    batch (`attempts_per_tick` attempts per call), where they share launches with each other. Two
    host threads drive the two batches on their own streams, so cheap requests are never held to
    the pace of an expensive one and the two batches' kernels overlap. policy "split_context":
    the expensive requests are instead solved one at a time on single-simulation contexts.
    order: "sjf" admits a batch lane's waiting requests shortest estimated work first, "fifo" in
    arrival order (a request that does not fit blocks the ones behind it); the context lane of
    split_context always takes its requests in arrival order. solo_max_steps > 0
    (policies split and split_context): a cheap request that finds its lane idle is solved at once
    on single-simulation contexts (_Lane.take_solo), so a lightly loaded server answers as fast as
    one request per launch."""

    def __init__(self, capacity_vortices: int, max_slots: int, attempts_per_tick: int = 4,
                 device: int = 0, keep_states: bool = False, policy: str = "fifo",
                 split_work: float = 2.0 ** 26, small_attempts: int = 16, order: str = "fifo",
                 expensive_fraction: float = 0.75, solo_max_steps: int = 0):
        if policy not in ("fifo", "split", "split_context"):
            raise ValueError("policy must be fifo, split or split_context")
        if order not in ("fifo", "sjf"):
            raise ValueError("order must be fifo or sjf")
        self.policy = policy
        self.order = order
        self.keep_states = keep_states
        self.split_work = split_work
        self.arrivals: list = []         # (arrival, rid, request) min-heap
        self.completions: list[Completion] = []
        if policy == "fifo":
            self.lanes = [_Lane(capacity_vortices, max_slots, device, attempts_per_tick)]
        elif policy == "split":
            # the arena (the HBM budget) is shared out: most room to the expensive requests
            big = int(capacity_vortices * expensive_fraction)
            self.lanes = [_Lane(capacity_vortices - big, max_slots, device, small_attempts,
                                solo_max_steps),
                          _Lane(big, max(max_slots // 4, 1), device, attempts_per_tick)]
        else:
            self.lanes = [_Lane(capacity_vortices, max_slots, device, small_attempts,
                                solo_max_steps),
                          _ContextLane(device, attempts_per_tick)]

    @property
    def batch(self) -> Batch:
        return self.lanes[0].batch

    def submit(self, req: Request) -> None:
        heapq.heappush(self.arrivals, (req.arrival, req.rid, req))

    def _lane_of(self, req: Request):
        if self.policy in ("split", "split_context") and work(req) > self.split_work:
            return self.lanes[1]
        return self.lanes[0]

    def _route(self, now: float) -> None:
        """Moves the requests that have arrived into their lane's ready list (arrival order, or
        shortest estimated work first with order "sjf")."""
        touched = set()
        while self.arrivals and self.arrivals[0][0] <= now:
            item = heapq.heappop(self.arrivals)
            lane = self._lane_of(item[2])
            lane.ready.append(item)
            touched.add(id(lane))
        if self.order == "sjf":
            # the context lane (split_context) keeps arrival order: it runs one request at a
            # time, and shortest-first there would hold the largest requests back without bound
            for lane in self.lanes:
                if id(lane) in touched and not isinstance(lane, _ContextLane):
                    lane.ready.sort(key=lambda it: (work(it[2]), it[0], it[1]))

    def _admit_lane(self, lane: _Lane, now: float) -> int:
        admitted = 0
        while lane.ready:
            _, _, req = lane.ready[0]
            x, y, g = req.state()
            try:
                sid = lane.batch.add(geometry_params(req.geometry), x, y, g, req.t_end,
                                     dt=req.dt, atol=req.atol, rtol=req.rtol,
                                     max_steps=req.max_steps)
            except CapacityError:
                break                   # wait for room: head-of-line, arrival order kept
            lane.ready.pop(0)
            lane.running[sid] = (req, now)
            admitted += 1
        return admitted

    def _admit(self, now: float) -> int:
        self._route(now)
        return sum(self._admit_lane(lane, now) for lane in self.lanes)

    def _retire(self, lane: _Lane, now: float, on_complete) -> int:
        done = 0
        for sid in list(lane.running):
            info = lane.batch.info(sid)
            if info.state == "running":
                continue
            req, _ = lane.running.pop(sid)
            x = y = None
            if self.keep_states or on_complete is not None:
                x, y = lane.batch.result(sid)
            lane.batch.release(sid)
            evals = 6 * (info.acceptedSteps + info.rejectedSteps) + 1
            c = Completion(req.rid, info.state, now - req.arrival, info.acceptedSteps, info.time,
                           x if self.keep_states else None, y if self.keep_states else None,
                           float(evals) * req.n * (req.n - 1))
            self.completions.append(c)
            if on_complete is not None:
                on_complete(c, x, y)
            done += 1
        return done

    def serve(self, requests: list[Request], on_complete: Optional[Callable] = None,
              clock=time.perf_counter) -> dict:
        """Runs the stream in real time: a request becomes visible at its arrival time. With
        policy "split" each batch is driven by its own host thread on its own CUDA stream, so the
        cheap requests' attempts run beside the expensive batch's instead of between them."""
        for r in requests:
            self.submit(r)
        start = clock()
        total = len(requests)
        if total == 0:
            pass
        elif self.policy in ("split", "split_context"):
            self._serve_threads(total, on_complete, clock, start)
        else:
            lane = self.lanes[0]
            while len(self.completions) < total:
                self._admit(clock() - start)
                if not lane.running:
                    if self.arrivals:
                        wait = self.arrivals[0][0] - (clock() - start)
                        if wait > 0:
                            time.sleep(min(wait, 0.01))
                    continue
                lane.batch.advance(lane.attempts)
                self._retire(lane, clock() - start, on_complete)
        elapsed = clock() - start
        out = summarize(self.completions, elapsed)
        out["policy"] = self.policy
        return out

    def _serve_threads(self, total: int, on_complete, clock, start: float) -> None:
        lock = threading.Lock()
        finished = threading.Event()
        errors: list = []

        def drive(lane) -> None:
            try:
                while not finished.is_set():
                    with lock:
                        self._route(clock() - start)
                        solo = lane.take_solo() if isinstance(lane, _Lane) else None
                        if solo is None:
                            lane.admit(self, clock() - start)
                        idle = not lane.running and solo is None
                        # sleep until the next arrival, at most 0.5 ms (another lane's arrival
                        # may be first)
                        nap = 0.0005
                        if self.arrivals:
                            nap = min(nap, max(0.0, self.arrivals[0][0] - (clock() - start)))
                    if solo is not None:
                        c, x, y = lane.run_solo(self, solo, clock, start, on_complete is not None)
                        with lock:
                            self.completions.append(c)
                            if on_complete is not None:
                                on_complete(c, x, y)
                            if len(self.completions) >= total:
                                finished.set()
                        continue
                    if idle:
                        time.sleep(nap)
                        continue
                    lane.advance()   # the GIL is released inside the library calls
                    with lock:
                        lane.retire(self, clock() - start, on_complete)
                        if len(self.completions) >= total:
                            finished.set()
            except BaseException as exc:  # surfaced to the caller below
                errors.append(exc)
                finished.set()

        threads = [threading.Thread(target=drive, args=(lane,), daemon=True) for lane in self.lanes]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        if errors:
            raise errors[0]

    def close(self):
        for lane in self.lanes:
            lane.close()


def summarize(completions: list[Completion], elapsed: float) -> dict:
    lat = np.array([c.latency for c in completions]) if completions else np.zeros(1)
    states = {}
    for c in completions:
        states[c.state] = states.get(c.state, 0) + 1
    engines = {}
    for c in completions:
        engines[c.engine] = engines.get(c.engine, 0) + 1
    pairs = sum(c.pairs for c in completions)
    return {"requests": len(completions), "elapsed_s": elapsed,
            "solves_per_s": len(completions) / elapsed if elapsed > 0 else 0.0,
            "pair_interactions_per_s": pairs / elapsed if elapsed > 0 else 0.0,
            "p50_latency_s": float(np.percentile(lat, 50)),
            "p99_latency_s": float(np.percentile(lat, 99)), "states": states,
            "engines": engines}


def one_at_a_time(requests: list[Request], device: int = 0, clock=time.perf_counter) -> dict:
    """FIFO baseline: each request solved alone through the single-simulation context API
    (pv_upload_state + pv_dopri5_step per step), in arrival order."""
    kernels = _contexts(device)
    out = []
    start = clock()
    for req in sorted(requests, key=lambda r: r.arrival):
        now = clock() - start
        if req.arrival > now:
            time.sleep(req.arrival - now)
        solver = _Solver(kernels, req)
        while not solver.step():
            pass
        out.append(Completion(req.rid, solver.state, clock() - start - req.arrival, solver.steps,
                              solver.t, pairs=solver.pairs(), engine="context"))
    for k in kernels.values():
        k.close()
    return summarize(out, clock() - start)
