"""The multi-GPU form of bench.py is N independent replicas: the job's step
time is the slowest rank's, the job's rate N steps per that time.  Tested
with two gloo ranks on the CPU (no GPU collective is involved)."""
import os
import socket

import pytest
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
        ms = [120.0, 180.0][rank]  # rank 1 is the slow replica
        ms_max = bench.slowest_rank(ms, world, "cpu")
        out[rank] = (ms_max, bench.job_rate(ms_max, world))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_replicas_take_the_slowest_rank():
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    for r in range(world):
        ms_max, rate = res[r]
        assert ms_max == 180.0
        assert rate == pytest.approx(2 * 1000.0 / 180.0)


def test_single_rank_is_its_own_time():
    import bench
    assert bench.slowest_rank(42.0, 1, "cpu") == 42.0
    assert bench.job_rate(500.0, 1) == 2.0
