"""The N > 1 path of bench.py on CPU: two gloo ranks, barrier + max-over-ranks.

The flux shards over ensemble members with no exchange, so multi-GPU runs are
independent replicas; the only collectives are the timing barrier and the
max reduction of the step time, which these ranks exercise without a GPU.
"""

import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, results):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench

    dist = bench.Dist()
    try:
        dist.barrier()
        # Each rank reports a different step time; every rank must see the max.
        results[rank] = dist.max(10.0 + rank)
        dist.barrier()
    finally:
        dist.close()


def test_two_rank_barrier_and_max():
    world = 2
    port = _free_port()
    with mp.Manager() as manager:
        results = manager.dict()
        mp.start_processes(_rank, args=(world, port, results), nprocs=world, start_method="spawn", join=True)
        assert dict(results) == {0: 11.0, 1: 11.0}
