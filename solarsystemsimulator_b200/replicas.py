"""Whole-job throughput of N independent replicas, one process per GPU.

The all-pairs path of one system does not shard here (one GPU per system;
the reference's multi-card target segmentation is not built), so
`bench.py --gpus N` runs N replicas of the same step. Each rank times its own
device work; the job took as long as its slowest rank, so the timing is the
maximum over ranks and the throughput is the units all ranks processed
divided by it. The reduction runs on whatever process group is initialised
(NCCL with a CUDA tensor on GPUs, gloo with a CPU tensor in the tests).
"""
from __future__ import annotations

import torch
import torch.distributed as dist


def max_over_ranks(x: float, device=None) -> float:
    """The maximum of x over all ranks (x itself without a process group)."""
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank: float, local_seconds: float, device=None) -> tuple[float, float]:
    """(units per second of the whole job, the slowest rank's seconds)."""
    world = dist.get_world_size() if dist.is_available() and dist.is_initialized() else 1
    t = max_over_ranks(local_seconds, device)
    if not t > 0.0:
        raise ValueError(f"job_rate: non-positive time {t}")
    return world * float(units_per_rank) / t, t
