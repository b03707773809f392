"""Image-level sharding for multi-GPU runs.

BM3D images are independent, so N GPUs split a batch of planes with no
collective on the data path: rank r filters a contiguous slice of the batch.
torch.distributed is used only for a barrier and the max-over-ranks time.
"""
from __future__ import annotations

from typing import List, Sequence, Tuple


def shard_range(n_items: int, rank: int, world: int) -> Tuple[int, int]:
    """[begin, end) of rank's contiguous slice; slices differ by at most one item."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    base, extra = divmod(n_items, world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def shard(items: Sequence, rank: int, world: int) -> List:
    b, e = shard_range(len(items), rank, world)
    return list(items[b:e])


def plane_seed(rank: int, set_index: int, plane_index: int) -> int:
    """Seed of a rank's synthetic plane: distinct across ranks, sets and planes."""
    return 1000 * rank + 100 * set_index + plane_index


def max_over_ranks(value: float, device=None) -> float:
    """Max of a per-rank scalar (a time) over the default process group;
    the value itself when not distributed."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
