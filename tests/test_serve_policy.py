"""Host-side logic of the serving loop, without a GPU: routing by estimated work, the batch lane's
shortest-first order against the context lane's arrival order, and when a request is solved
alone (solo). The lanes are built without their device objects."""
from pointvortex_b200.serve import Request, Server, _ContextLane, _Lane, work


def _lane(solo_max_steps=0):
    lane = object.__new__(_Lane)
    lane.ready, lane.running = [], {}
    lane.solo_max_steps = solo_max_steps
    lane.kernels = {} if solo_max_steps > 0 else None
    return lane


def _context_lane():
    lane = object.__new__(_ContextLane)
    lane.ready, lane.running, lane.current = [], {}, None
    return lane


def _server(policy="split_context", order="sjf", split_work=2.0 ** 20):
    s = object.__new__(Server)
    s.policy, s.order, s.split_work = policy, order, split_work
    s.arrivals, s.completions, s.keep_states = [], [], False
    s.lanes = [_lane(16), _context_lane()]
    return s


def _req(rid, geometry, n, arrival, max_steps=10):
    return Request(rid, geometry, n, 1, 0.1, 1e-9, max_steps=max_steps, arrival=arrival)


def test_routing_by_work_and_lane_orders():
    s = _server()
    reqs = [_req(0, "periodic", 4000, 0.0), _req(1, "infinite", 900, 0.1),
            _req(2, "periodic", 3000, 0.2), _req(3, "infinite", 100, 0.3),
            _req(4, "disk", 300, 0.4)]
    for r in reqs:
        s.submit(r)
    s._route(0.25)  # the first three have arrived
    cheap, expensive = s.lanes
    assert [it[2].rid for it in expensive.ready] == [0, 2]      # arrival order
    assert [it[2].rid for it in cheap.ready] == [1]
    s._route(1.0)
    assert [it[2].rid for it in cheap.ready] == [3, 4, 1]       # shortest estimated work first
    assert work(reqs[3]) < work(reqs[4]) < work(reqs[1])
    assert [it[2].rid for it in expensive.ready] == [0, 2]


def test_solo_only_for_an_idle_lane_with_one_budgeted_request():
    lane = _lane(16)
    assert lane.take_solo() is None                              # nothing waiting
    lane.ready = [(0.0, 1, _req(1, "infinite", 100, 0.0, max_steps=10))]
    lane.running = {7: None}
    assert lane.take_solo() is None                              # the batch is busy
    lane.running = {}
    assert lane.take_solo().rid == 1 and lane.ready == []        # idle, alone, budget <= 16
    lane.ready = [(0.0, 2, _req(2, "infinite", 100, 0.0, max_steps=40))]
    assert lane.take_solo() is None                              # budget above the limit
    lane.ready = [(0.0, 3, _req(3, "infinite", 100, 0.0, max_steps=0))]
    assert lane.take_solo() is None                              # no budget: runs to t_end
    lane.ready = [(0.0, 4, _req(4, "infinite", 100, 0.0)), (0.0, 5, _req(5, "infinite", 90, 0.0))]
    assert lane.take_solo() is None                              # two waiting: batch them
    assert _lane(0).take_solo() is None                          # solo off
