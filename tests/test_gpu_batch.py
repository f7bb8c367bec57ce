"""Batched ensembles: one persistent launch per RK stage over members of
uneven sizes must give every member exactly what it gets when run alone."""
import numpy as np
import pytest

from chimera_b200 import problems as P
from chimera_b200.config import BC_OUTFLOW, FP32_BULK
from tests.gpu_util import require_gpu

pytestmark = pytest.mark.gpu


def _members(precision=0):
    out = []
    for k, n in enumerate([40, 64, 37, 96, 64, 128]):
        cfg, st = P.grf_member(n, 100 + k)
        if k == 2:   # a ragged outflow member among periodic ones
            cfg = cfg.replace(bc=(BC_OUTFLOW,) * 4)
        out.append((cfg.replace(precision=precision), st))
    return out


@pytest.fixture(scope="module")
def G():
    return require_gpu()


def test_fp64_batch_matches_oracle_per_member(G, oracle):
    mem = _members()
    s = G.Solver([c for c, _ in mem])
    for m, (_, st) in enumerate(mem):
        s.set_state(st, member=m)
    s.step(12)
    for m, (cfg, st) in enumerate(mem):
        ref = oracle.State(st)
        dts = oracle.run(cfg, ref, 12)
        out = s.get_state(member=m)
        for q in range(6):
            assert np.array_equal(out[q], ref.a[q]), (m, q)
        d = s.diag(member=m)
        assert d["t"] == ref.t and d["steps"] == 12


def test_fp32_batch_matches_single_grid_runs(G):
    mem = _members(FP32_BULK)
    s = G.Solver([c for c, _ in mem])
    for m, (_, st) in enumerate(mem):
        s.set_state(st, member=m)
    s.step(10)
    for m, (cfg, st) in enumerate(mem):
        one = G.Solver(cfg)
        one.set_state(st)
        one.step(10)
        for x, y in zip(s.get_state(member=m), one.get_state()):
            assert np.array_equal(x, y), m
        one.close()


def test_batch_graph_replay(G):
    mem = _members(FP32_BULK)
    a = G.Solver([c for c, _ in mem])
    b = G.Solver([c for c, _ in mem])
    for m, (_, st) in enumerate(mem):
        a.set_state(st, member=m)
        b.set_state(st, member=m)
    a.step(6)
    b.set_graph_steps(3)
    b.step(3)
    b.step(3)
    for m in range(len(mem)):
        for x, y in zip(a.get_state(member=m), b.get_state(member=m)):
            assert np.array_equal(x, y)


def test_batch_members_stop_independently(G, oracle):
    """Members with different t_end stop at their own times (device-side)."""
    mem = _members()[:3]
    cfgs = [c.replace(t_end=te) for (c, _), te in zip(mem, (0.004, 0.012, 0.02))]
    s = G.Solver(cfgs)
    for m, (_, st) in enumerate(mem):
        s.set_state(st, member=m)
    s.advance()
    for m, ((_, st), cfg) in enumerate(zip(mem, cfgs)):
        ref = oracle.State(st)
        oracle.run(cfg, ref, 100000)
        d = s.diag(member=m)
        assert d["active"] == 0 and d["t"] == ref.t
        for x, y in zip(s.get_state(member=m), ref.a):
            assert np.array_equal(x, y)


def test_batch_autotune_and_variants(G, oracle):
    mem = _members()
    s = G.Solver([c for c, _ in mem])
    for m, (_, st) in enumerate(mem):
        s.set_state(st, member=m)
    s.autotune(reps=1)
    s.step(4)
    cfg, st = mem[3]
    ref = oracle.State(st)
    oracle.run(cfg, ref, 4)
    for x, y in zip(s.get_state(member=3), ref.a):
        assert np.array_equal(x, y)
