"""Ensembles across GPUs as replicas: the cost partition, and the gathering of every rank's
results on rank 0 over a two-rank gloo group (the engine itself stubbed: no GPU here)."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from pointvortex_b200.shard import partition, run_sharded, simulation_cost, torch_gather


def test_partition_balances_and_is_deterministic():
    rng = np.random.default_rng(3)
    specs = [(("infinite", "periodic", "disk")[k % 3], int(np.exp(rng.uniform(np.log(64), np.log(8192)))))
             for k in range(512)]
    costs = [simulation_cost(g, n) for g, n in specs]
    for world in (2, 4, 8):
        owner = partition(costs, world)
        assert owner == partition(costs, world)
        loads = np.zeros(world)
        for c, r in zip(costs, owner):
            loads[r] += c
        # longest-processing-time: every rank within the largest single cost of the mean
        assert loads.max() - loads.min() <= max(costs)
        assert set(owner) == set(range(world))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        specs = [("periodic", 100 + 37 * k) for k in range(23)]
        merged = run_sharded(specs, lambda s: simulation_cost(*s),
                             lambda mine: [(i, (rank, s[1] * 2)) for i, s in mine],
                             rank, world, torch_gather)
        out[rank] = merged
    finally:
        dist.destroy_process_group()


def test_results_gather_on_rank_zero_over_gloo():
    world = 2
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    assert res[1] is None
    merged = res[0]
    assert [m[1] for m in merged] == [2 * (100 + 37 * k) for k in range(23)]
    assert {m[0] for m in merged} == {0, 1}   # both ranks did work
