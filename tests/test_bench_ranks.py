"""The multi-rank logic of bench.py on CPU: two gloo ranks (world size 2),
each with its own step time; every rank must see the maximum, and the
whole-job rate counts the units of all ranks over that maximum."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import bench
    local = [3.5, 4.25][rank]
    worst = bench.max_over_ranks(local, dist, "cpu")
    dist.barrier()
    out[rank] = worst
    dist.destroy_process_group()


def test_max_over_ranks_with_two_gloo_ranks():
    world = 2
    port = _free_port()
    out = mp.Manager().dict()
    mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
    assert out[0] == out[1] == 4.25


def test_whole_job_rate_and_single_rank():
    import bench
    assert bench.max_over_ranks(2.0) == 2.0
    # 2 ranks x 1000 fluid x 10 steps in 0.5 s
    assert bench.whole_job_rate(1000, 10, 2, 0.5) == pytest.approx(40000.0)
