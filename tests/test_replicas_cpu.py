"""Replica timing of bench.py on two gloo ranks (CPU): every rank reports
its own device time, the job time is the maximum over ranks, and the rate is
the whole job's (world x steps over that time).  The same functions run over
NCCL on the GPUs."""
import os
import socket
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        ms = bench.max_over_ranks(100.0 + 25.0 * rank, world, "cpu")
        dist.barrier()
        out[rank] = (ms, bench.replica_rate(world, 5, ms))
    finally:
        dist.destroy_process_group()


def test_two_rank_max_and_rate():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0] == res[1]
    ms, rate = res[0]
    assert ms == 125.0
    assert rate == pytest.approx(2 * 5 / 0.125)


def test_single_rank_passthrough():
    import bench
    assert bench.max_over_ranks(42.0, 1, "cpu") == 42.0
    assert bench.replica_rate(1, 3, 1000.0) == pytest.approx(3.0)
