"""The replica aggregation of `bench.py --gpus N` (apbs_b200/replicas.py)
across two gloo ranks on the CPU: the job's rate is every rank's
calculations over the slowest rank's time."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from apbs_b200 import replicas


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mx, sm = replicas.torch_reducers(dist, torch.device("cpu"))
        # rank r ran 10 + r calculations in 100 * (r + 1) ms
        rate, ms = replicas.aggregate(10.0 + rank, 100.0 * (rank + 1), mx, sm)
        out[rank] = (rate, ms)
    finally:
        dist.destroy_process_group()


def test_two_ranks_sum_units_over_slowest_time():
    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    # 21 calculations over the slower rank's 200 ms, the same on both ranks
    for rank in range(world):
        rate, ms = res[rank]
        assert ms == 200.0
        assert rate == pytest.approx(21.0 / 0.2)


def test_single_rank_is_the_local_rate():
    ident = lambda x: x
    rate, ms = replicas.aggregate(5, 50.0, ident, ident)
    assert ms == 50.0 and rate == pytest.approx(100.0)
