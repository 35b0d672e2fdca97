"""One process per GPU: the rank plumbing of multi-GPU runs.

Pixels are independent, so ranks share no data on the inversion's path: each
rank inverts its own pixels with its own plan, and the only collectives are
the barriers around timed regions, the max-over-ranks reduction of their
times, and gathering results where one process writes them.  The process
group is NCCL on GPUs (torch.distributed, one process per GPU, launched by
torchrun) and gloo on the CPU (the tests).
"""
from __future__ import annotations

import datetime
import os


def rank_env():
    """(rank, world size, local rank) from the launcher's environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", timeout_s: int = 600, device=None):
    """The process group when there is more than one rank, else None."""
    rank, world, _ = rank_env()
    if world <= 1:
        return None
    import torch.distributed as dist
    kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
    if device is not None:
        kw["device_id"] = device
    dist.init_process_group(backend, **kw)
    return dist


def map_seed(rank: int, base: int = 1000) -> int:
    """Seed of a rank's own synthetic map (weak scaling: one map per rank)."""
    return base + rank


def shard(total: int, rank: int, world: int):
    """Contiguous pixel range [start, start + count) of a rank when the ranks
    split one map (strong scaling): sizes differ by at most one pixel."""
    base, extra = divmod(total, world)
    start = rank * base + min(rank, extra)
    return start, base + (1 if rank < extra else 0)


def _reduce(x: float, dist, op_name: str, device) -> float:
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=getattr(dist.ReduceOp, op_name))
    return float(t.item())


def max_over_ranks(x: float, dist, device="cpu") -> float:
    """The slowest rank's time (every rank gets it)."""
    return _reduce(x, dist, "MAX", device)


def sum_over_ranks(x: float, dist, device="cpu") -> float:
    return _reduce(x, dist, "SUM", device)


def gather_rows(rows, dist, world: int, device="cpu"):
    """Concatenation in rank order of every rank's rows (numpy [n][k]), on
    every rank; ranks may hold different n."""
    import numpy as np
    if dist is None:
        return rows
    import torch
    out = [None] * world
    dist.all_gather_object(out, np.asarray(rows))
    return np.concatenate(out)
