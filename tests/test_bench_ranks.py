"""bench.py at N > 1 ranks (replicas, one per GPU): every rank times its own
replica and the job's time is the maximum over ranks.  The reduction is
checked here with two gloo ranks on the CPU."""
import os
import socket

import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        out[rank] = bench.max_over_ranks(1.5 + rank, world)
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        assert dict(out) == {0: 2.5, 1: 2.5}


def test_max_over_ranks_single_rank():
    import bench
    assert bench.max_over_ranks(3.25, 1) == 3.25
