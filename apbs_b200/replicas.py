"""Whole-job throughput of independent replicas.

The PMG solve does not shard: `bench.py --gpus N` runs one calculation stream
per GPU (one process per GPU under torchrun) with no data exchange between
them.  The job's throughput is the calculations all ranks finished over the
slowest rank's device time, the two reductions below; the ranks pass their
collective (NCCL on GPUs, gloo in the CPU test) as plain functions.
"""
from __future__ import annotations

from typing import Callable


def aggregate(local_units: float, local_ms: float, reduce_max: Callable[[float], float],
              reduce_sum: Callable[[float], float]) -> tuple[float, float]:
    """(units per second over all ranks, the slowest rank's milliseconds)."""
    total_ms = reduce_max(local_ms)
    total_units = reduce_sum(local_units)
    return total_units / (total_ms / 1e3), total_ms


def torch_reducers(dist, device) -> tuple[Callable[[float], float], Callable[[float], float]]:
    """max and sum over the ranks of a torch.distributed process group."""
    import torch

    def red(x: float, op) -> float:
        t = torch.tensor([x], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=op)
        return float(t.item())

    return (lambda x: red(x, dist.ReduceOp.MAX)), (lambda x: red(x, dist.ReduceOp.SUM))
