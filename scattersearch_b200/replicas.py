"""Multi-GPU execution: independent replicas with host-side query sharding.

Queries are independent and every GPU holds a full copy of the index, so the
path shards by query with no device collective (sharding the index instead
would change the traversal and the ids).  Each rank searches a contiguous
range of the query set; results come back to rank 0 through one host-side
gather.  Timings are reduced as the maximum over ranks.
"""
from __future__ import annotations

import numpy as np


def shard_range(n: int, rank: int, world: int):
    """Contiguous [start, end) of n items for `rank` of `world`; sizes differ
    by at most one and the ranges tile [0, n) in rank order."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def gather_rows(local: np.ndarray, n_total: int, rank: int, world: int, group=None):
    """Concatenates each rank's contiguous shard (rows of equal width) on
    every rank, in rank order, through torch.distributed all_gather_object
    (host-side; any backend)."""
    import torch.distributed as dist
    if world == 1:
        return local
    parts = [None] * world
    dist.all_gather_object(parts, local, group=group)
    out = np.concatenate(parts, axis=0)
    if out.shape[0] != n_total:
        raise RuntimeError(f"gathered {out.shape[0]} rows, expected {n_total}")
    return out


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of a per-rank float (e.g. elapsed seconds) over all ranks."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
