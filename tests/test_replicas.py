"""The multi-GPU form of the benchmark is independent replicas: each rank runs its own simulation
and the only cross-rank step is the final reduction of the figures (max of the device times, sum
of the pairs). Two gloo ranks on the CPU check that reduction and that the reference arm runs on
rank 0 alone."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    import bench
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms, pairs = bench.combine_ranks(10.0 + 5.0 * rank, 1e6 * (rank + 1))
        ref = bench.run_reference(type("A", (), {"steps": 1, "warmup": 0})()) if rank else None
        out[rank] = (ms, pairs, ref)
    finally:
        dist.destroy_process_group()


def test_replica_figures_reduce_over_two_gloo_ranks():
    world = 2
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    for rank in range(world):
        ms, pairs, ref = res[rank]
        assert ms == 15.0                      # the slowest rank's device time
        assert pairs == 3e6                    # every rank's pairs
    assert res[1][2] is None                   # the reference arm does no work off rank 0


def test_single_process_combine_is_identity():
    import bench
    assert bench.combine_ranks(3.0, 7.0) == (3.0, 7.0)
