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


# Per-member diagnostics gathered across ranks (the fields of chimera_diag_out).
DIAG_FIELDS = ("t", "dt", "steps", "divb_max", "divb_mean", "bmax", "divb_rel", "mass", "energy",
               "cfl_speed", "mood_resets", "floor_hits", "status")
_INT_FIELDS = {"steps", "mood_resets", "floor_hits", "status"}


def gather_member_rows(rows, n_members: int, width: int, group=None, device=None):
    """Every member's row of ``width`` float64 values, on every rank.

    Each rank passes ``{global member index: row}`` for the members it
    advances (``shard_members``); the rows go into a table of zeros that is
    summed across the ranks of ``group``.  Every member is owned by exactly one
    rank, so the sum is a gather (x + 0.0 == x, up to the sign of a zero).  It
    is the one collective of a sharded ensemble and carries diagnostics, never
    state.  Without an initialised process group the local table is returned.
    ``device`` must suit the backend (a CUDA device for NCCL)."""
    import torch
    import torch.distributed as dist
    t = torch.zeros((n_members, width), dtype=torch.float64, device=device)
    for m, row in rows.items():
        if not 0 <= m < n_members:
            raise ValueError(f"member {m} outside 0..{n_members - 1}")
        t[m] = torch.as_tensor(row, dtype=torch.float64, device=t.device)
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(t, group=group)
    return t


def gather_diagnostics(solver, members, n_members: int, group=None, device=None):
    """Every member's diagnostics on every rank: a list, indexed by global
    member, of dicts with ``DIAG_FIELDS``.  ``solver`` holds this rank's
    members in the order of ``members`` (their global indices) and answers
    ``diag(member=k)`` like ``gpu.Solver``."""
    rows = {}
    for k, m in enumerate(members):
        d = solver.diag(member=k)
        rows[m] = [float(d[f]) for f in DIAG_FIELDS]
    table = gather_member_rows(rows, n_members, len(DIAG_FIELDS), group, device).cpu().tolist()
    return [{f: (int(v) if f in _INT_FIELDS else v) for f, v in zip(DIAG_FIELDS, r)} for r in table]
