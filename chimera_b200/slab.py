"""One grid split into y-slabs across ranks (one process per GPU).

The reference advances one grid in one process (src/main.f90:65-303).  Here
rank r of W holds the grid rows [y0, y1) (a near-equal split) plus GHOST ghost
rows on each side that has a neighbour; a side without one (the grid's own
non-periodic edge) keeps the grid's boundary condition.  One step on every
rank:

    pack the interior rows the neighbours need -> exchange -> unpack into the
    ghost rows -> CFL dt of the slab's own rows -> minimum over the ranks ->
    the three RK3 stages (chimera_step)

(the slab's dt for the next step comes from its stage-3 epilogue, which
leaves the ghost rows out, so no separate CFL pass runs after the first step)

Why GHOST = 7: the slab's ghost sides are declared outflow, and what that
boundary does to the outer ghost rows spreads two rows per RK3 stage (slopes
and MOOD bounds reach one row beyond a face's two cells).  At the bottom the
lowest ghost row is wrong before the first stage: its cell-centred B
averages the face below it (src/mhd_field_ops.f90:120-156), which the slab
does not hold.  So after the three stages rows 0..6 from the bottom and
0..5 from the top may differ from the undivided grid's; with seven ghost
rows every interior cell, and the face b_y below the lowest interior cell,
is bit-for-bit the undivided grid's.  (Six rows are not enough:
tests/test_slab.py shows it.)

The dt is exact: the CFL reductions of each slab (its stage-3 epilogue and
the CFL pass) cover only its own rows (chimera_slab_ghost_rows), whose
values after a step are already the undivided grid's, the slabs' rows
partition the grid, and the dt is a minimum (src/main.f90:72-83, the tOut
clip is monotone), so the minimum over the slabs is the grid's dt.

The exchange moves 2 x GHOST x nx x 6 values per slab and step (1.4 MB per
side in FP64 at nx = 4096); nothing else crosses ranks.  Diagnostics
(``SlabSolver.diag``: div B, |B|, totals over the slab's own rows) combine
across ranks by max / sum.

Transports: ``DistTransport`` (torch.distributed: NCCL between GPUs, gloo
between CPU processes) for one slab per process, ``LocalTransport`` for
several slabs in one process (copies; no slab waits on another's kernels).
"""
from __future__ import annotations

import contextlib
from dataclasses import dataclass

import numpy as np
import torch

from .config import BC_OUTFLOW, BC_PERIODIC, FP32_BULK, SolverConfig

GHOST = 7


def slab_rows(ny: int, world: int, rank: int):
    """Rows [y0, y1) of rank ``rank``: ny split into ``world`` near-equal
    contiguous slabs, the first ny % world one row taller."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("bad world/rank")
    base, extra = divmod(ny, world)
    y0 = rank * base + min(rank, extra)
    return y0, y0 + base + (1 if rank < extra else 0)


@dataclass
class SlabLayout:
    rank: int
    world: int
    y0: int
    y1: int
    lo: int                 # ghost rows below the slab (0 at the grid's own lower edge)
    hi: int                 # ghost rows above
    lo_peer: int | None     # rank holding the rows below, or None
    hi_peer: int | None
    cfg: SolverConfig       # the slab's grid: ny = interior + lo + hi
    ny_global: int

    @property
    def interior(self) -> int:
        return self.y1 - self.y0

    def global_rows(self) -> np.ndarray:
        """Grid row of every local row (periodic wrap for the ghost rows)."""
        return np.arange(self.y0 - self.lo, self.y1 + self.hi) % self.ny_global


def slab_layout(cfg: SolverConfig, world: int, rank: int, ghost: int = GHOST) -> SlabLayout:
    """The slab of rank ``rank`` of ``world`` for the grid ``cfg``."""
    py = cfg.bc[2] == BC_PERIODIC
    if py != (cfg.bc[3] == BC_PERIODIC):
        raise ValueError("periodic y needs both y sides periodic")
    if ghost < 1:
        raise ValueError("ghost must be >= 1")
    y0, y1 = slab_rows(cfg.ny, world, rank)
    if world == 1:
        return SlabLayout(rank, world, y0, y1, 0, 0, None, None, cfg, cfg.ny)
    if y1 - y0 < ghost:
        raise ValueError(f"a slab of {y1 - y0} rows is thinner than its {ghost} ghost rows")
    has_lo = rank > 0 or py
    has_hi = rank < world - 1 or py
    lo, hi = (ghost if has_lo else 0), (ghost if has_hi else 0)
    bc = (cfg.bc[0], cfg.bc[1], BC_OUTFLOW if has_lo else cfg.bc[2], BC_OUTFLOW if has_hi else cfg.bc[3])
    local = cfg.replace(ny=(y1 - y0) + lo + hi, bc=bc)
    return SlabLayout(rank, world, y0, y1, lo, hi,
                      (rank - 1) % world if has_lo else None,
                      (rank + 1) % world if has_hi else None, local, cfg.ny)


class SlabSolver:
    """Rank ``rank``'s slab of the grid ``cfg`` on the current CUDA device.

    Its kernels, and the exchange of ``slab_step``, run on one torch stream
    (``stream``, default a new one): the slabs of one process share it, so
    that packing, copying and unpacking are ordered without events."""

    def __init__(self, cfg: SolverConfig, rank: int = 0, world: int = 1, ghost: int = GHOST,
                 stream: "torch.cuda.Stream | None" = None):
        from .gpu import Solver
        self.layout = slab_layout(cfg, world, rank, ghost)
        self.ghost = ghost
        self.stream = stream if stream is not None else torch.cuda.Stream()
        self.solver = Solver([self.layout.cfg], stream=self.stream.cuda_stream)
        if self.layout.lo or self.layout.hi:
            self.solver.slab_ghost_rows(self.layout.lo, self.layout.hi)
        store = torch.float32 if cfg.precision == FP32_BULK else torch.float64
        shape = (6, ghost, cfg.nx)
        lo, hi = self.layout.lo, self.layout.hi
        self.send_lo = torch.empty(shape, dtype=store, device="cuda") if lo else None
        self.recv_lo = torch.empty(shape, dtype=store, device="cuda") if lo else None
        self.send_hi = torch.empty(shape, dtype=store, device="cuda") if hi else None
        self.recv_hi = torch.empty(shape, dtype=store, device="cuda") if hi else None
        self.dt = torch.zeros(1, dtype=torch.float64, device="cuda")

    def set_global_state(self, arrays, t: float = 0.0, output_count: int = 1):
        """Take this slab's rows (with ghost rows) of the six grid arrays
        (Mass, Momx, Momy, Energy, b_x, b_y; (ny, nx), host or device)."""
        idx = torch.as_tensor(self.layout.global_rows())
        self.stream.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(self.stream):
            local = []
            for a in arrays:
                a = torch.as_tensor(a)
                local.append(a.index_select(0, idx.to(a.device)).to(device="cuda", dtype=torch.float64).contiguous())
            self.solver.set_state(local)
            self.solver.set_time(t, output_count)

    def interior_state(self):
        """The slab's own rows of the state, six (interior, nx) numpy arrays."""
        full = self.solver.get_state()
        lo = self.layout.lo
        return [a[lo:lo + self.layout.interior] for a in full]

    def diag(self) -> dict:
        """CFL dt, div B, |B| and totals of the slab's own rows for the
        current state (synchronises): max / sum them over the ranks."""
        self.solver.refresh_dt()
        return self.solver.diag()

    # the per-step pieces (asynchronous on the stream)
    def pack(self):
        if self.send_lo is not None or self.send_hi is not None:
            self.solver.halo_pack(self.ghost, self.send_lo, self.send_hi)

    def unpack(self):
        if self.recv_lo is not None or self.recv_hi is not None:
            self.solver.halo_unpack(self.ghost, self.recv_lo, self.recv_hi)

    def refresh_dt(self):
        # the dt the last stage 3 computed over the slab's own rows (a CFL pass
        # before the first step); the ghost-row unpack does not change it
        self.solver.get_dt_device(self.dt)

    def set_dt(self):
        self.solver.set_dt_device(self.dt)

    def step_local(self):
        self.solver.step(1)

    def close(self):
        self.solver.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
        return False


class LocalTransport:
    """All slabs in this process: ghost rows and dt by device copies."""

    def exchange(self, slabs):
        by_rank = {s.layout.rank: s for s in slabs}
        for s in slabs:
            L = s.layout
            if L.lo_peer is not None:
                s.recv_lo.copy_(by_rank[L.lo_peer].send_hi)
            if L.hi_peer is not None:
                s.recv_hi.copy_(by_rank[L.hi_peer].send_lo)

    def min_dt(self, slabs):
        m = torch.min(torch.cat([s.dt for s in slabs])).reshape(1)
        for s in slabs:
            s.dt.copy_(m)


class DistTransport:
    """One slab per process over torch.distributed (the default group's ranks).

    Sends go out in a fixed order (to the upper neighbour, then to the lower
    one) and receives are posted in the matching order (from the lower
    neighbour, then from the upper one), with tags naming the receiving side:
    with two ranks and periodic y both neighbours are the same rank, and a
    backend that matches messages in order (NCCL) or by tag (gloo) pairs them
    the same way."""

    TO_LO_GHOST, TO_HI_GHOST = 0, 1

    def __init__(self, group=None):
        self.group = group

    def exchange(self, slabs):
        import torch.distributed as dist
        (s,) = slabs
        L = s.layout
        ops = []
        if L.hi_peer is not None:
            ops.append(dist.P2POp(dist.isend, s.send_hi, L.hi_peer, self.group, self.TO_LO_GHOST))
        if L.lo_peer is not None:
            ops.append(dist.P2POp(dist.isend, s.send_lo, L.lo_peer, self.group, self.TO_HI_GHOST))
        if L.lo_peer is not None:
            ops.append(dist.P2POp(dist.irecv, s.recv_lo, L.lo_peer, self.group, self.TO_LO_GHOST))
        if L.hi_peer is not None:
            ops.append(dist.P2POp(dist.irecv, s.recv_hi, L.hi_peer, self.group, self.TO_HI_GHOST))
        if ops:
            for r in dist.batch_isend_irecv(ops):
                r.wait()

    def min_dt(self, slabs):
        import torch.distributed as dist
        (s,) = slabs
        dist.all_reduce(s.dt, op=dist.ReduceOp.MIN, group=self.group)


def _on_stream(slabs):
    st = getattr(slabs[0], "stream", None)
    if st is None:                        # slabs without a device stream
        return contextlib.nullcontext()
    if any(getattr(s, "stream", None) != st for s in slabs):
        raise ValueError("the slabs of one process must share one stream")
    return torch.cuda.stream(st)


def slab_step(slabs, transport, nsteps: int = 1):
    """Advance every slab in ``slabs`` (this process's) by ``nsteps`` RK3
    steps, exchanging ghost rows and dt through ``transport`` each step.
    Every rank calls it with the same ``nsteps``."""
    with _on_stream(slabs):
        _steps(slabs, transport, int(nsteps))


def _steps(slabs, transport, nsteps):
    for _ in range(nsteps):
        for s in slabs:
            s.pack()
        transport.exchange(slabs)
        for s in slabs:
            s.unpack()
            s.refresh_dt()
        transport.min_dt(slabs)
        for s in slabs:
            s.set_dt()
            s.step_local()


def gather_interior(slabs):
    """The grid's six arrays assembled from the slabs of one process (all
    ranks present), in rank order."""
    parts = [s.interior_state() for s in sorted(slabs, key=lambda s: s.layout.rank)]
    return [np.concatenate([p[q] for p in parts], axis=0) for q in range(6)]


__all__ = ["GHOST", "slab_rows", "SlabLayout", "slab_layout", "SlabSolver", "LocalTransport", "DistTransport",
           "slab_step", "gather_interior"]
