"""Frame sharding across ranks (one process per GPU).

Frames never interact (src/batch.rs:69-101), so a batch is split into
contiguous, balanced per-rank shards integrated by each rank's own plan
replica; the only collective is the max over ranks of the device-timed
elapsed time (and, on request, gathering results on one rank). No collective
sits on the data path.
"""
from __future__ import annotations


def shard(n_items: int, rank: int, world: int) -> tuple:
    """[start, stop) of rank's contiguous share of n_items; the first
    n_items % world ranks take one item more."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    if n_items < 0:
        raise ValueError("item count must not be negative")
    base, extra = divmod(n_items, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def max_over_ranks(value: float, device=None) -> float:
    """The maximum of value over all ranks of the default process group
    (the value itself without one)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
