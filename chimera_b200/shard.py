"""Sharding of independent ensemble members across ranks (one process per GPU).

Members never exchange data, so the only cross-rank traffic is timing and
diagnostics (max / sum reductions); there is no data-path collective.
"""
from __future__ import annotations


def shard_members(cells_per_member, world: int, rank: int):
    """Indices of the members rank ``rank`` of ``world`` advances: greedy
    longest-processing-time assignment by cell count (largest member first to
    the least-loaded rank; ties to the lowest rank), deterministic on every
    rank.  Returns the indices in increasing order."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("bad world/rank")
    load = [0] * world
    owner = [0] * len(cells_per_member)
    order = sorted(range(len(cells_per_member)), key=lambda m: (-cells_per_member[m], m))
    for m in order:
        r = min(range(world), key=lambda k: (load[k], k))
        owner[m] = r
        load[r] += cells_per_member[m]
    return [m for m in range(len(cells_per_member)) if owner[m] == rank]


def shard_loads(cells_per_member, world: int):
    return [sum(cells_per_member[m] for m in shard_members(cells_per_member, world, r)) for r in range(world)]
