"""The y-slab decomposition of one grid (chimera_b200.slab) on CPU: the slab
layout, and the per-step exchange + dt minimum driven by the package's own
``slab_step`` and transports, with each slab advanced by the CPU oracle
(the GPU slabs run the same driver; tests/test_gpu_slab.py).  Interior
cells must equal the undivided grid's bit for bit."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from chimera_b200 import problems
from chimera_b200.config import BC_OUTFLOW, BC_PERIODIC
from chimera_b200.slab import (GHOST, DistTransport, LocalTransport, slab_layout, slab_rows,
                               slab_step)


class OracleSlab:
    """A slab with the interface of ``SlabSolver``, advanced by the CPU oracle."""

    def __init__(self, cfg, rank, world, ghost=GHOST):
        from oracle import oracle as O
        self.O = O
        self.layout = slab_layout(cfg, world, rank, ghost)
        self.ghost = ghost
        nx = cfg.nx
        mk = lambda need: torch.zeros((6, ghost, nx), dtype=torch.float64) if need else None  # noqa: E731
        self.send_lo, self.recv_lo = mk(self.layout.lo), mk(self.layout.lo)
        self.send_hi, self.recv_hi = mk(self.layout.hi), mk(self.layout.hi)
        self.dt = torch.zeros(1, dtype=torch.float64)

    def set_global_state(self, arrays, t=0.0, output_count=1):
        rows = self.layout.global_rows()
        self.state = self.O.State([np.asarray(a)[rows] for a in arrays], t, output_count)

    def pack(self):
        G, ny = self.ghost, self.layout.cfg.ny
        for q in range(6):
            if self.send_lo is not None:
                self.send_lo[q] = torch.from_numpy(self.state.a[q][G:2 * G])
            if self.send_hi is not None:
                self.send_hi[q] = torch.from_numpy(self.state.a[q][ny - 2 * G:ny - G])

    def unpack(self):
        G, ny = self.ghost, self.layout.cfg.ny
        for q in range(6):
            if self.recv_lo is not None:
                self.state.a[q][0:G] = self.recv_lo[q].numpy()
            if self.recv_hi is not None:
                self.state.a[q][ny - G:ny] = self.recv_hi[q].numpy()

    def refresh_dt(self):
        # the CFL minimum over the slab's own rows (the ghost rows are left out)
        c = self.layout.cfg
        lo, n = self.layout.lo, self.layout.interior
        prims = [np.ascontiguousarray(p[lo:lo + n]) for p in self.O.primitives(c, self.state.a)]
        self.dt[0] = self.O.cfl_dt(c.replace(ny=n), *prims, t=self.state.t, output_count=self.state.output_count)

    def set_dt(self):
        self._dt = float(self.dt[0])

    def step_local(self):
        self.O.run(self.layout.cfg, self.state, 1, dt_fixed=[self._dt])

    def interior_state(self):
        lo = self.layout.lo
        return [a[lo:lo + self.layout.interior] for a in self.state.a]


def _assemble(slabs):
    parts = [s.interior_state() for s in sorted(slabs, key=lambda s: s.layout.rank)]
    return [np.concatenate([p[q] for p in parts], axis=0) for q in range(6)]


def _whole(oracle, cfg, st, nsteps):
    s = oracle.State(st)
    oracle.run(cfg, s, nsteps)
    return s


# ---- layout ---------------------------------------------------------------------

@pytest.mark.parametrize("ny,world", [(256, 1), (256, 8), (100, 7), (13, 2)])
def test_rows_cover_the_grid_once(ny, world):
    rows = [slab_rows(ny, world, r) for r in range(world)]
    assert rows[0][0] == 0 and rows[-1][1] == ny
    assert all(rows[r][1] == rows[r + 1][0] for r in range(world - 1))
    sizes = [b - a for a, b in rows]
    assert max(sizes) - min(sizes) <= 1


def test_layout_periodic_and_outflow():
    cfg, _ = problems.orszag_tang(48)
    L = [slab_layout(cfg, 3, r) for r in range(3)]
    assert [(x.lo, x.hi) for x in L] == [(GHOST, GHOST)] * 3
    assert [(x.lo_peer, x.hi_peer) for x in L] == [(2, 1), (0, 2), (1, 0)]
    assert all(x.cfg.bc[2:] == (BC_OUTFLOW, BC_OUTFLOW) and x.cfg.bc[:2] == cfg.bc[:2] for x in L)
    assert list(L[0].global_rows()[:GHOST]) == list(range(48 - GHOST, 48))
    rcfg, _ = problems.rotor(48)
    R = [slab_layout(rcfg, 3, r) for r in range(3)]
    assert [(x.lo, x.hi) for x in R] == [(0, GHOST), (GHOST, GHOST), (GHOST, 0)]
    assert (R[0].lo_peer, R[2].hi_peer) == (None, None)
    assert R[0].cfg.ny == 16 + GHOST and R[1].cfg.ny == 16 + 2 * GHOST
    one = slab_layout(cfg, 1, 0)
    assert (one.lo, one.hi, one.cfg) == (0, 0, cfg)


def test_layout_rejects():
    cfg, _ = problems.orszag_tang(16)
    with pytest.raises(ValueError):
        slab_layout(cfg, 4, 0)              # 4-row slabs, 7 ghost rows
    with pytest.raises(ValueError):
        slab_layout(cfg.replace(bc=(BC_PERIODIC, BC_PERIODIC, BC_PERIODIC, BC_OUTFLOW)), 2, 0)
    with pytest.raises(ValueError):
        slab_layout(cfg, 2, 2)


# ---- one process, several slabs ----------------------------------------------------

def _local_run(cfg, st, world, nsteps, ghost=GHOST):
    slabs = [OracleSlab(cfg, r, world, ghost) for r in range(world)]
    for s in slabs:
        s.set_global_state(st)
    slab_step(slabs, LocalTransport(), nsteps)
    return slabs


@pytest.mark.parametrize("case", ["ot_periodic_4", "ot_periodic_2", "rotor_outflow_3", "field_loop_dxdy_3"])
def test_local_slabs_equal_the_whole_grid(oracle, case):
    if case.startswith("ot"):
        cfg, st = problems.orszag_tang(48)
        world = int(case[-1])
    elif case.startswith("rotor"):
        cfg, st = problems.rotor(48)
        world = 3
    else:
        cfg, st = problems.field_loop(nx=32, ny=40)
        world = 3
    nsteps = 6
    slabs = _local_run(cfg, st, world, nsteps)
    got = _assemble(slabs)
    ref = _whole(oracle, cfg, st, nsteps)
    for q in range(6):
        assert np.array_equal(got[q], ref.a[q]), q
    assert all(s.state.t == ref.t and s.state.output_count == ref.output_count for s in slabs)


def test_fewer_ghost_rows_are_not_enough(oracle):
    """Six ghost rows let the lower boundary reach the first interior row
    within one step (its lowest ghost row is wrong before the first stage):
    seven is the smallest exact width."""
    cfg, st = problems.orszag_tang(48)
    st = _whole(oracle, cfg, st, 2).a
    ref = _whole(oracle, cfg, st, 1)
    exact = _assemble(_local_run(cfg, st, 4, 1, ghost=7))
    short = _assemble(_local_run(cfg, st, 4, 1, ghost=6))
    assert all(np.array_equal(exact[q], ref.a[q]) for q in range(6))
    assert any(not np.array_equal(short[q], ref.a[q]) for q in range(6))


# ---- gloo ranks ---------------------------------------------------------------------

def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, kind, nsteps, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    cfg, st = problems.orszag_tang(48) if kind == "ot" else problems.rotor(48)
    s = OracleSlab(cfg, rank, world)
    s.set_global_state(st)
    slab_step([s], DistTransport(), nsteps)
    out.put((rank, [a.copy() for a in s.interior_state()], s.state.t))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("kind,world", [("ot", 2), ("rotor", 3)])
def test_gloo_ranks_equal_the_whole_grid(oracle, kind, world):
    """World 2 with periodic y: both neighbours are the same rank (the
    ordering / tag rule of DistTransport); world 3 outflow: edge slabs with
    one ghost side."""
    nsteps = 4
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, kind, nsteps, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=180) for _ in range(world)], key=lambda x: x[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    cfg, st = problems.orszag_tang(48) if kind == "ot" else problems.rotor(48)
    ref = _whole(oracle, cfg, st, nsteps)
    for qf in range(6):
        got = np.concatenate([r[1][qf] for r in res], axis=0)
        assert np.array_equal(got, ref.a[qf]), qf
    assert all(r[2] == ref.t for r in res)


def _leaving_worker(rank, world, port, leave_rank, steps_before, out):
    """Rank ``leave_rank`` leaves after ``steps_before`` steps, between steps
    and with nothing in flight; the others go on stepping."""
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    cfg, st = problems.orszag_tang(48)
    s = OracleSlab(cfg, rank, world)
    s.set_global_state(st)
    try:
        slab_step([s], DistTransport(), steps_before)
        if rank == leave_rank:
            out.put((rank, "left"))
            out.close()
            out.join_thread()
            os._exit(3)
        slab_step([s], DistTransport(), 2)
        out.put((rank, "finished"))
    except Exception:   # the failure this test expects on the remaining ranks
        out.put((rank, "error"))
        out.close()
        out.join_thread()
        os._exit(4)


def test_a_rank_that_leaves_ends_the_others_exchange_with_an_error():
    """Failure detection on the host: when one slab's rank exits between
    steps, the other rank's next ghost-row exchange (or dt minimum) ends with
    an error within the process group's timeout instead of waiting for good."""
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_leaving_worker, args=(r, world, port, 1, 2, q)) for r in range(world)]
    for p in procs:
        p.start()
    try:
        res = dict(q.get(timeout=120) for _ in range(world))
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert res == {0: "error", 1: "left"}
    assert procs[0].exitcode == 4 and procs[1].exitcode == 3
