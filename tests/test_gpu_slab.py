"""One grid split into y-slabs (chimera_b200.slab) on one GPU: the slabs are
separate handles stepped in turn on one stream, their ghost rows and dt moved
by device copies (LocalTransport) -- no slab's kernels wait on another's.
Interior cells must equal the undivided grid's bit for bit, in FP64 and in
the FP32-bulk form, and the per-slab diagnostics must combine to the grid's."""
import numpy as np
import pytest
import torch

from chimera_b200 import problems as P
from chimera_b200.config import FP32_BULK, HLLD, HLLE
from chimera_b200.slab import GHOST, LocalTransport, SlabSolver, gather_interior, slab_step
from tests.gpu_util import require_gpu

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def G():
    return require_gpu()


def _whole(G, cfg, st, nsteps):
    s = G.Solver(cfg)
    s.set_state(st)
    s.step(nsteps)
    out = s.get_state()
    d = s.diag()
    s.close()
    return out, d


def _slabs(cfg, st, world, nsteps):
    stream = torch.cuda.Stream()
    slabs = [SlabSolver(cfg, r, world, stream=stream) for r in range(world)]
    for s in slabs:
        s.set_global_state(st)
    slab_step(slabs, LocalTransport(), nsteps)
    return slabs


CASES = {
    "ot256_periodic_4": (lambda: P.orszag_tang(256), 4, 20),
    "ot128_periodic_2": (lambda: P.orszag_tang(128), 2, 20),        # both neighbours the same slab
    "rotor200_outflow_3": (lambda: P.rotor(200, riemann=HLLE), 3, 20),
    "kh192_hlld_5": (lambda: P.kelvin_helmholtz(192, riemann=HLLD), 5, 15),
    "field_loop_96x150_3": (lambda: P.field_loop(96, 150), 3, 15),
}


@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("fp32", [False, True])
def test_slabs_equal_the_whole_grid(G, case, fp32):
    make, world, nsteps = CASES[case]
    cfg, st = make()
    if fp32:
        cfg = cfg.replace(precision=FP32_BULK)
    ref, dref = _whole(G, cfg, st, nsteps)
    slabs = _slabs(cfg, st, world, nsteps)
    got = gather_interior(slabs)
    for q in range(6):
        assert np.array_equal(got[q], ref[q]), q
    ds = [s.diag() for s in slabs]
    assert all(d["t"] == dref["t"] and d["steps"] == nsteps for d in ds)
    # the next step's dt, max |div B| and max |B| are maxima / minima: exact
    assert min(d["dt"] for d in ds) == dref["dt"]
    assert max(d["divb_max"] for d in ds) == dref["divb_max"]
    assert max(d["bmax"] for d in ds) == dref["bmax"]
    assert sum(d["mass"] for d in ds) == pytest.approx(dref["mass"], rel=1e-13)
    assert sum(d["energy"] for d in ds) == pytest.approx(dref["energy"], rel=1e-13)
    for s in slabs:
        s.close()


def test_six_ghost_rows_differ(G):
    """The GPU path has the reach the CPU test measures: six rows are not enough."""
    cfg, st = P.orszag_tang(128)
    ref, _ = _whole(G, cfg, st, 3)
    stream = torch.cuda.Stream()
    short = [SlabSolver(cfg, r, 4, ghost=GHOST - 1, stream=stream) for r in range(4)]
    for s in short:
        s.set_global_state(st)
    slab_step(short, LocalTransport(), 3)
    got = gather_interior(short)
    assert any(not np.array_equal(got[q], ref[q]) for q in range(6))


def test_halo_rows_round_trip(G):
    """pack -> unpack through the C-ABI moves exactly the documented rows."""
    cfg, st = P.orszag_tang(64)
    s = G.Solver(cfg)
    s.set_state(st)
    rows = 5
    lo = torch.empty((6, rows, 64), dtype=torch.float64, device="cuda")
    hi = torch.empty_like(lo)
    s.halo_pack(rows, lo, hi)
    torch.cuda.synchronize()
    for q in range(6):
        assert np.array_equal(lo[q].cpu().numpy(), st[q][rows:2 * rows])
        assert np.array_equal(hi[q].cpu().numpy(), st[q][64 - 2 * rows:64 - rows])
    s.halo_unpack(rows, hi, lo)        # swap: rows [0,5) <- hi pack, rows [59,64) <- lo pack
    out = s.get_state()
    for q in range(6):
        assert np.array_equal(out[q][:rows], st[q][64 - 2 * rows:64 - rows])
        assert np.array_equal(out[q][64 - rows:], st[q][rows:2 * rows])
        assert np.array_equal(out[q][rows:64 - rows], st[q][rows:64 - rows])
    s.close()


def test_halo_rejects_bad_arguments(G):
    cfg, st = P.orszag_tang(32)
    s = G.Solver(cfg)
    buf = torch.empty((6, 20, 32), dtype=torch.float64, device="cuda")
    for rows in (0, 17):
        with pytest.raises(G.ChimeraError):
            s.halo_pack(rows, buf, None)
    with pytest.raises(G.ChimeraError):
        s.slab_ghost_rows(16, 16)
    s.close()
    b = G.Solver([cfg, cfg])
    with pytest.raises(G.ChimeraError):
        b.halo_pack(2, buf, None)
    b.close()


def test_slab_steps_take_dt_from_the_fused_epilogue(G):
    """After the first step a slab's dt comes from its stage-3 epilogue (which
    leaves the ghost rows out): one CFL kernel launch in all, and still the
    undivided grid's result."""
    cfg, st = P.orszag_tang(128)
    ref, _ = _whole(G, cfg, st, 6)
    stream = torch.cuda.Stream()
    slabs = [SlabSolver(cfg, r, 3, stream=stream) for r in range(3)]
    for s in slabs:
        s.set_global_state(st)
        s.solver.set_profiling(True)
    slab_step(slabs, LocalTransport(), 6)
    prof = [s.solver.get_profile() for s in slabs]
    assert all(p["cfl"]["launches"] == 1 and p["stage3"]["launches"] == 6 for p in prof)
    got = gather_interior(slabs)
    assert all(np.array_equal(got[q], ref[q]) for q in range(6))
    for s in slabs:
        s.close()
