"""Continuous batching: requests that arrive while others are on the GPU are admitted as room frees
up, and every result is the same as the request solved alone."""
import numpy as np
import pytest

from pointvortex_b200.batch import Batch, geometry_params
from pointvortex_b200.serve import Request, Server, one_at_a_time, poisson_stream

pytestmark = pytest.mark.gpu


def alone(req: Request):
    b = Batch(max(req.n, 2) + 512, 1)
    x, y, g = req.state()
    sid = b.add(geometry_params(req.geometry), x, y, g, req.t_end, dt=req.dt, atol=req.atol,
                rtol=req.rtol, max_steps=req.max_steps)
    b.run()
    info = b.info(sid)
    out = b.result(sid)
    b.close()
    return info, out


def test_stream_results_equal_alone_results():
    reqs = poisson_stream(24, rate=400.0, seed=3, n_min=32, n_max=1500, t_end_range=(0.01, 0.03),
                          rtols=(1e-6, 1e-9), max_steps=40)
    # a small arena forces queueing: later requests wait for earlier ones to retire
    server = Server(capacity_vortices=4000, max_slots=6, attempts_per_tick=2, keep_states=True)
    streamed = []
    summary = server.serve(reqs, on_complete=lambda c, x, y: streamed.append(c.rid))
    server.close()
    assert summary["requests"] == len(reqs) == len(streamed)
    assert summary["p99_latency_s"] >= summary["p50_latency_s"] > 0
    by_id = {c.rid: c for c in server.completions}
    overlapped = 0
    for req in reqs:
        c = by_id[req.rid]
        info, (x, y) = alone(req)
        assert c.state == info.state and c.accepted_steps == info.acceptedSteps, req
        assert np.array_equal(c.x, x) and np.array_equal(c.y, y), req
        overlapped += 1
    assert overlapped == len(reqs)


def test_one_at_a_time_baseline_agrees():
    reqs = poisson_stream(4, rate=1000.0, seed=5, n_min=64, n_max=600, t_end_range=(0.005, 0.01),
                          rtols=(1e-8,), max_steps=30)
    s = one_at_a_time(reqs)
    assert s["requests"] == 4
    for req in reqs:
        info, _ = alone(req)
        assert info.state in ("done", "budget", "failed")


def alone_on_a_context(req: Request):
    from pointvortex_b200.serve import _contexts, _Solver
    kernels = _contexts(0)
    solver = _Solver(kernels, req)
    while not solver.step():
        pass
    return solver.state, solver.steps, solver.positions()


def _serve_split(policy: str, order: str):
    reqs = poisson_stream(16, rate=400.0, seed=11, n_min=32, n_max=3000, t_end_range=(0.01, 0.02),
                          rtols=(1e-6, 1e-9), max_steps=30)
    server = Server(capacity_vortices=20000, max_slots=8, attempts_per_tick=2, keep_states=True,
                    policy=policy, split_work=2.0 ** 18, small_attempts=4, order=order)
    summary = server.serve(reqs)
    server.close()
    assert summary["requests"] == len(reqs) and summary["policy"] == policy
    return reqs, server


def test_split_policy_results_equal_alone_results():
    """Admission by estimated work (cheap and expensive requests in two batches, two threads and
    streams, shortest estimated work first) changes when a request runs, never what it computes:
    every result equals the request solved alone in a batch of its own."""
    reqs, server = _serve_split("split", "sjf")
    by_id = {c.rid: c for c in server.completions}
    expensive = 0
    for req in reqs:
        c = by_id[req.rid]
        expensive += server._lane_of(req) is server.lanes[1]
        info, (x, y) = alone(req)
        assert c.state == info.state and c.accepted_steps == info.acceptedSteps, req
        assert np.array_equal(c.x, x) and np.array_equal(c.y, y), req
        assert c.pairs > 0
    assert 0 < expensive < len(reqs)


def test_split_context_policy_results_equal_alone_results():
    """The variant with the expensive requests on single-simulation contexts, one at a time."""
    from pointvortex_b200.serve import _ContextLane
    reqs, server = _serve_split("split_context", "fifo")
    by_id = {c.rid: c for c in server.completions}
    on_contexts = 0
    for req in reqs:
        c = by_id[req.rid]
        if isinstance(server._lane_of(req), _ContextLane):
            on_contexts += 1
            state, steps, (x, y) = alone_on_a_context(req)
            assert c.state == state and c.accepted_steps == steps, req
        else:
            info, (x, y) = alone(req)
            assert c.state == info.state and c.accepted_steps == info.acceptedSteps, req
        assert np.array_equal(c.x, x) and np.array_equal(c.y, y), req
        assert c.pairs > 0
    assert 0 < on_contexts < len(reqs)


def test_idle_cheap_requests_are_solved_alone_on_contexts():
    """solo_max_steps: a cheap request that finds its lane idle and alone in its queue is solved at
    once on single-simulation contexts (the same result as alone on a context); requests that
    arrive together are batched (the same result as alone in a batch)."""
    reqs = poisson_stream(10, rate=60.0, seed=13, n_min=32, n_max=800, t_end_range=(0.01, 0.02),
                          rtols=(1e-6, 1e-9), max_steps=12)
    # two requests at the same instant: they cannot both go solo
    reqs[5].arrival = reqs[4].arrival
    server = Server(capacity_vortices=20000, max_slots=8, attempts_per_tick=2, keep_states=True,
                    policy="split", split_work=2.0 ** 30, small_attempts=4, order="sjf",
                    solo_max_steps=16)
    streamed = []
    summary = server.serve(reqs, on_complete=lambda c, x, y: streamed.append((c.rid, x is not None)))
    server.close()
    assert summary["requests"] == len(reqs) == len(streamed)
    assert all(has_state for _, has_state in streamed)
    by_id = {c.rid: c for c in server.completions}
    engines = set()
    for req in reqs:
        c = by_id[req.rid]
        engines.add(c.engine)
        if c.engine == "context":
            state, steps, (x, y) = alone_on_a_context(req)
            assert c.state == state and c.accepted_steps == steps, req
        else:
            info, (x, y) = alone(req)
            assert c.state == info.state and c.accepted_steps == info.acceptedSteps, req
        assert np.array_equal(c.x, x) and np.array_equal(c.y, y), req
    assert "context" in engines
    # a request with a budget above solo_max_steps never goes solo
    big = poisson_stream(1, rate=10.0, seed=14, n_min=32, n_max=64, max_steps=40)
    server = Server(capacity_vortices=20000, max_slots=8, policy="split", solo_max_steps=16)
    server.serve(big)
    server.close()
    assert server.completions[0].engine == "batch"
