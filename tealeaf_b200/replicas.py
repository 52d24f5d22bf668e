"""Whole-job throughput of independent replicas (one process per GPU).

The solver path does not shard (one chunk per GPU, no halo exchange, no
collective on the data path): N ranks each run the same timesteps on their
own GPU. The only communication is this aggregation after the timed region:
the job's time is the slowest rank's device time, its work the sum of the
ranks' iterations. Works with any torch.distributed backend (nccl on GPUs,
gloo on the CPU for tests).
"""
from __future__ import annotations

from typing import Tuple


def aggregate(ms: float, iterations: float, world: int, device: str = "cuda") -> Tuple[float, float]:
    """(max over ranks of ms, sum over ranks of iterations); identity when world == 1."""
    if world <= 1:
        return float(ms), float(iterations)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(ms), float(iterations)], dtype=torch.float64, device=device)
    mx, sm = t.clone(), t.clone()
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    dist.all_reduce(sm, op=dist.ReduceOp.SUM)
    return mx[0].item(), sm[1].item()


def throughput(ms: float, iterations: float, world: int, device: str = "cuda") -> float:
    """Job iterations per second: summed iterations over the slowest rank's time."""
    ms_max, its = aggregate(ms, iterations, world, device)
    return its / (ms_max / 1000.0)
