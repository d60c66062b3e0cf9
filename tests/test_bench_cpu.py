"""CPU: the replica aggregation of bench.py under torch.distributed (gloo, two ranks).

Multi-GPU runs of the bench are replicas: each rank solves its own copy and the job's time
is the maximum over ranks; the whole-job rate counts every rank's solves.  The GPU part of
the bench needs a B200; the rank logic runs here on gloo."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = 100.0 * (rank + 1)  # rank 1 is the slow one
        m = bench.replica_max(ms, world, "cpu")
        out[rank] = (m, bench.replica_throughput(world, 5, m))
    finally:
        dist.destroy_process_group()


def test_replica_max_and_throughput_over_gloo_ranks():
    world = 2
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    # every rank sees the slowest rank's time; 2 ranks x 5 solves in 0.2 s
    assert res[0] == res[1] == (200.0, 50.0)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.replica_max(12.5, 1, "cpu") == 12.5
    assert bench.replica_throughput(1, 4, 200.0) == 20.0
