"""Multi-GPU bookkeeping of the chain: one process per GPU, no data-path collective.

A-scans are independent, so a volume shards into contiguous B-scan ranges,
one per rank, each processed by that rank's own context; outputs are written
per rank (the host gathers them if one buffer spans GPUs). The only
collective is the timing reduction of a benchmark: the maximum over ranks of
the device time, from which the whole-job throughput is computed.
torch.distributed carries it (NCCL on GPUs, gloo on CPU for the tests).
"""
from __future__ import annotations

from typing import Optional, Tuple


def bscan_range(total_bscans: int, world: int, rank: int) -> Tuple[int, int]:
    """(first B-scan, count) of `rank` when `total_bscans` are split as evenly
    as possible into `world` contiguous ranges (the first ranks take one more)."""
    if world < 1 or not 0 <= rank < world or total_bscans < 0:
        raise ValueError("need world >= 1, 0 <= rank < world and total_bscans >= 0")
    base, extra = divmod(total_bscans, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of `value` over all ranks of the default process group (the
    value itself without one). `device` is where the reduction tensor lives:
    a CUDA device for NCCL, None (CPU) for gloo."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def weak_scaling_rate(units_per_rank: float, seconds_max: float, world: int) -> float:
    """Whole-job throughput when every rank processes `units_per_rank` units
    and the slowest rank takes `seconds_max`."""
    if seconds_max <= 0:
        raise ValueError("seconds_max must be positive")
    return world * units_per_rank / seconds_max


def rank_setup(env: Optional[dict] = None) -> Tuple[int, int, int]:
    """(world size, rank, local rank) from the torchrun environment."""
    import os
    e = os.environ if env is None else env
    return int(e.get("WORLD_SIZE", "1")), int(e.get("RANK", "0")), int(e.get("LOCAL_RANK", "0"))
