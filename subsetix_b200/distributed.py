"""Sharding of independent work across ranks (one process per GPU).

Everything on this path is row-local: sets, expressions, AMR fields of
independent simulations.  A global batch is therefore split into
contiguous shards, one per rank, and each rank evaluates its shard with no
data-path collective.  The only communication is the timing reduction,
which takes the maximum over ranks (the job's time is its slowest rank's).
"""

from __future__ import annotations

from typing import Tuple


def shard(total: int, rank: int, world: int) -> Tuple[int, int]:
    """``(first, count)`` of rank ``rank``'s contiguous share of ``total`` units (sizes differ by at most one)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must lie in [0, world)")
    if total < 0:
        raise ValueError("total must be non-negative")
    base, extra = divmod(int(total), int(world))
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def max_over_ranks(value: float, device=None) -> float:
    """The maximum of ``value`` over the ranks of the default process group (the value itself when there is none)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


__all__ = ["shard", "max_over_ranks"]
