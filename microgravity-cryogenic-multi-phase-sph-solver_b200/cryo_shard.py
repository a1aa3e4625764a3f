"""Sharding independent tanks over ranks (one process per GPU).

Tanks of an ensemble share nothing during a step, so a multi-GPU ensemble is
a partition of the tanks with no collective in the data path: each rank
builds and steps its own shard, and the per-tank results are gathered once
at the end.  The partition is longest-processing-time first on the particle
count (a tank's step cost grows with its particles): tanks in decreasing
size, each to the currently least-loaded rank (ties to the lower rank).
"""
from __future__ import annotations

from typing import Dict, List, Sequence


def lpt_shards(sizes: Sequence[int], world: int) -> List[List[int]]:
    """Tank indices per rank; every index appears exactly once."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(sizes)), key=lambda t: (-int(sizes[t]), t))
    shards: List[List[int]] = [[] for _ in range(world)]
    load = [0] * world
    for t in order:
        r = min(range(world), key=lambda k: (load[k], k))
        shards[r].append(t)
        load[r] += max(int(sizes[t]), 1)
    return shards


def shard_of(sizes: Sequence[int], rank: int, world: int) -> List[int]:
    return lpt_shards(sizes, world)[rank]


def gather_per_tank(local: Dict[int, object], group=None) -> Dict[int, object]:
    """All ranks' {tank index: result} merged on every rank (one
    all_gather_object over the process group; a host-side exchange after the
    run, not a data-path collective)."""
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized():
        return dict(local)
    parts: List[Dict[int, object]] = [None] * dist.get_world_size(group)  # type: ignore[list-item]
    dist.all_gather_object(parts, local, group=group)
    out: Dict[int, object] = {}
    for p in parts:
        for k, v in p.items():
            if k in out:
                raise RuntimeError(f"tank {k} reported by two ranks")
            out[k] = v
    return out
