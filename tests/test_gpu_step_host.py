"""chimera_step_host: one step on host arrays, in row bands -- the inputs land
band by band under the CFL kernel, the stages run as a wavefront over the
bands (stage 1 on band k, stage 2 on k - 1, stage 3 on k - 2) where y is not
periodic, and stage 3's finished bands go back while later bands compute.  It
must give exactly what set_state + step + get_state give."""
import numpy as np
import pytest
import torch

from chimera_b200 import problems as P
from chimera_b200.config import BC_OUTFLOW, BC_PERIODIC, FP32_BULK
from tests.gpu_util import require_gpu

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def G():
    return require_gpu()


def _reference_steps(G, cfg, st, n):
    s = G.Solver(cfg)
    out, states = st, []
    for _ in range(n):
        s.set_state(out)
        s.step(1)
        out = s.get_state()
        states.append((out, s.diag()))
    s.close()
    return states


def _pinned(arrays):
    return [torch.from_numpy(np.ascontiguousarray(a)).pin_memory() for a in arrays]


@pytest.mark.parametrize("case", ["rotor128", "rotor512", "ragged50x37", "ot96"])
def test_step_host_equals_set_step_get(G, case):
    if case.startswith("rotor"):
        cfg, st = P.rotor(int(case[5:]))
    elif case == "ragged50x37":
        cfg, st = P.orszag_tang(50)
        cfg = cfg.replace(bc=(BC_PERIODIC, BC_PERIODIC, BC_OUTFLOW, BC_OUTFLOW))
        st = [a[:37].copy() for a in st]
        cfg = cfg.replace(ny=37)
    else:
        cfg, st = P.orszag_tang(96)
    ref = _reference_steps(G, cfg, st, 3)
    s = G.Solver(cfg)
    buf = _pinned(st)
    for k in range(3):
        s.step_host(buf, out=buf)                 # in place, pinned
        for q in range(6):
            assert np.array_equal(buf[q].numpy(), ref[k][0][q]), (k, q)
        d = s.diag()
        assert (d["t"], d["dt"], d["output_count"]) == (ref[k][1]["t"], ref[k][1]["dt"], ref[k][1]["output_count"])
    s.close()


def test_step_host_then_device_steps(G):
    """After step_host the handle holds the new state and its dt: device steps continue from it."""
    cfg, st = P.rotor(64)
    a = G.Solver(cfg)
    a.set_state(st)
    a.step(3)
    b = G.Solver(cfg)
    b.step_host(st)
    b.step(2)
    for x, y in zip(a.get_state(), b.get_state()):
        assert np.array_equal(x, y)


def test_step_host_inactive_returns_input(G):
    cfg, st = P.orszag_tang(32, t_end=0.5)
    s = G.Solver(cfg)
    s.set_time(0.6, 61)
    out = s.step_host(st)
    for x, y in zip(out, st):
        assert np.array_equal(x, y)


def test_step_host_fp32_handle(G):
    cfg, st = P.orszag_tang(64)
    c32 = cfg.replace(precision=FP32_BULK)
    ref = _reference_steps(G, c32, st, 2)
    s = G.Solver(c32)
    out = st
    for k in range(2):
        out = s.step_host(out)
        for q in range(6):
            assert np.array_equal(out[q], ref[k][0][q])


@pytest.mark.parametrize("fp32", [False, True])
def test_set_state_has_read_pinned_arrays_on_return(G, fp32):
    """set_state from page-locked host tensors: the caller may overwrite them
    as soon as the call returns (host arrays are read completely before it
    returns), and get_state gives back exactly what was set."""
    cfg, st = P.rotor(1024)   # 48 MB of state: a copy still in flight would be seen
    if fp32:
        cfg = cfg.replace(precision=FP32_BULK)
    s = G.Solver(cfg)
    pinned = _pinned(st)
    s.set_state(pinned)
    for t in pinned:
        t.fill_(float("nan"))
    got = s.get_state()
    ref = G.Solver(cfg)       # the same arrays set from pageable numpy memory
    ref.set_state(st)
    want = ref.get_state()    # FP32-bulk: the set values rounded to FP32
    ref.close()
    s.close()
    for a, b in zip(got, want):
        assert np.array_equal(a, b)
