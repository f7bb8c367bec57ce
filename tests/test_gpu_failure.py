"""Failure detection without faulting the GPU: non-finite states reach the
device status word and come back as CHIMERA_ERR_NONFINITE; finished runs stop
on the device; floors keep a near-vacuum cell finite."""
import numpy as np
import pytest

from chimera_b200 import problems as P
from tests.gpu_util import require_gpu

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def G():
    return require_gpu()


def test_nan_seeded_cell_sets_status(G):
    cfg, st = P.orszag_tang(64)
    st[3] = st[3].copy()
    st[3][10, 20] = np.nan
    s = G.Solver(cfg)
    s.set_state(st)
    s.step(2)
    d = s.diag()
    assert d["status"] != 0
    with pytest.raises(G.ChimeraError) as e:
        s.get_state()
    assert e.value.code == -3
    out = s.get_state(check=False)          # still copied out
    assert np.isnan(out[3]).any()


def test_inactive_after_t_end_leaves_state(G):
    cfg, st = P.orszag_tang(32, t_end=0.01)
    s = G.Solver(cfg)
    s.set_state(st)
    n = s.advance()
    a = s.get_state()
    s.step(5)                                # t >= t_end: kernels skip on the device
    b = s.get_state()
    d = s.diag()
    assert n > 0 and d["active"] == 0 and d["steps"] == n
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_near_vacuum_cell_floored_and_finite(G, oracle):
    cfg, st = P.rotor(64)
    st[0] = st[0].copy()
    st[0][30, 30] = 1e-20 * cfg.dx * cfg.dy   # density far below the 1e-12 floor
    s = G.Solver(cfg)
    s.set_state(st)
    s.set_counters(True)
    s.step(5)
    out = s.get_state()
    d = s.diag()
    assert d["status"] == 0 and d["floor_hits"] > 0
    assert all(np.isfinite(x).all() for x in out)
    ref = oracle.State(st)
    oracle.run(cfg, ref, 5)
    for x, y in zip(out, ref.a):
        assert np.array_equal(x, y)


def test_bad_arguments_rejected(G):
    cfg, st = P.orszag_tang(16)
    s = G.Solver(cfg)
    with pytest.raises(ValueError):
        s.set_state([a[:, :8] for a in st])
    with pytest.raises(G.ChimeraError):
        s.stage(4, 1e-3)
    with pytest.raises(G.ChimeraError):
        s.set_variant(99)


def test_handles_close_at_the_end_of_a_with_block(G):
    """Solver and Adjoint free their C handles on leaving a with block, an
    exception included."""
    import torch

    from chimera_b200.adjoint import Adjoint
    cfg, st = P.orszag_tang(32)
    with G.Solver(cfg) as s:
        s.set_state(st)
        s.step(1)
        assert s.handle
    assert not s.handle
    with pytest.raises(RuntimeError):
        with G.Solver(cfg) as s2:
            raise RuntimeError("inside the block")
    assert not s2.handle
    with Adjoint(cfg) as a:
        U = [torch.from_numpy(x.copy()).cuda() for x in st]
        a.forward_step(U, 1e-3)
    assert not a._h
