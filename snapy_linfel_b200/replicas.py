"""Multi-GPU plumbing of the replica runs: one process per GPU, no exchange on
the data path.

The single-domain step shards by slab decomposition with a ghost exchange per
stage (layout.py); an ensemble shards trivially by whole members.  These
helpers give the rank geometry, the max-over-ranks device timing every
multi-rank number uses, and a size-balanced assignment of ensemble members to
ranks.
"""
from __future__ import annotations

import os


def rank_info():
    """(rank, world, local_rank) from the launcher's environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def max_over_ranks(value: float, device="cpu") -> float:
    """The maximum of a per-rank number (a timed duration) over all ranks."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device="cpu") -> float:
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def shard_members(sizes, world: int):
    """Assign members (by cell count) to `world` ranks, largest first onto the
    least loaded rank; returns one sorted index list per rank."""
    loads = [0] * world
    out = [[] for _ in range(world)]
    for m in sorted(range(len(sizes)), key=lambda k: (-sizes[k], k)):
        r = min(range(world), key=lambda q: (loads[q], q))
        out[r].append(m)
        loads[r] += sizes[m]
    return [sorted(x) for x in out]
