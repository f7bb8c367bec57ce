"""GRF ensembles of uneven grid sizes, advanced as one batch (one persistent
launch per RK stage over every member's tiles).

Replaces the reference's sequential ensemble driver
(``scripts/run_mhd_MC.py:57-78``: one process per seed).  Members are
independent; they share the solver switches and precision of the batch.
"""
from __future__ import annotations

from . import problems
from .config import FP32_BULK, FP64


def grf_ensemble(scale: int = 1, precision: int = FP32_BULK, seed0: int = 1000, members=None):
    """Configs and conserved states of the GRF ensemble: 256 members at 128^2,
    192 at 256^2, 64 at 512^2 (``scale`` divides the member counts).  Member k
    is seeded with ``seed0 + k`` (Philox).  ``members`` selects a subset of
    member indices (a rank's shard)."""
    cfgs, states = [], []
    sizes = problems.grf_ensemble_sizes(scale)
    for k, n in enumerate(sizes):
        if members is not None and k not in members:
            continue
        cfg, st = problems.grf_member(n, seed0 + k)
        cfgs.append(cfg.replace(precision=precision))
        states.append(st)
    return cfgs, states


def make_batch(cfgs, states, gpu_module=None):
    """A batched solver holding every member's state."""
    if gpu_module is None:
        from . import gpu as gpu_module
    s = gpu_module.Solver(cfgs)
    try:
        for m, st in enumerate(states):
            s.set_state(st, member=m)
    except BaseException:
        s.close()
        raise
    return s


def cells(cfgs) -> int:
    return sum(c.nx * c.ny for c in cfgs)


__all__ = ["grf_ensemble", "make_batch", "cells", "FP64", "FP32_BULK"]
