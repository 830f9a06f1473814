"""Replica aggregation for multi-GPU runs.

The render path has no exchange step (pixels, samples and views are independent), so N
GPUs run N independent replicas. The only cross-rank work is the measurement: every rank
reports its samples and device seconds, and the job's throughput is all samples over the
slowest rank's time. Works with any torch.distributed backend (nccl on GPUs, gloo in tests).
"""
from __future__ import annotations

from typing import Optional, Tuple

import torch
import torch.distributed as dist


def aggregate(samples: float, seconds: float, hops: float = 0.0,
              device: Optional[torch.device] = None) -> Tuple[float, float, float]:
    """Returns (total samples, max seconds, total hops) over all ranks; identity when the
    process group is not initialised."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(samples), float(seconds), float(hops)
    dev = device or torch.device("cpu")
    t = torch.tensor([seconds], dtype=torch.float64, device=dev)
    tot = torch.tensor([samples, hops], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(tot, op=dist.ReduceOp.SUM)
    return float(tot[0].item()), float(t.item()), float(tot[1].item())


def replica_seed(global_seed: int, rank: int) -> int:
    """Per-rank seed so replicas render different sample sets of the same frame."""
    return (global_seed + 7919 * rank) & 0xFFFFFFFF
