"""chimera_rk3_step_noalloc: one RK3 step that allocates no device memory.

Callers whose device memory is owned entirely by their own allocator, or whose
time loop must not pay cudaMalloc's implicit device synchronisation, use this
entry point instead of a handle.  It must give the same bits as the handle path
(chimera_create / chimera_step) -- the FP64 tolerance of these tests is exact
equality -- on consecutive calls that reuse the shared scratch array.

This file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from chimera_b200 import problems as P
from chimera_b200.config import HLLD, HLLE, RUSANOV
from tests.gpu_util import require_gpu

pytestmark = pytest.mark.gpu


def _noalloc(G):
    L = G.lib()
    f = L.chimera_rk3_step_noalloc
    f.argtypes = [C.POINTER(G.CCfg)] + [C.c_void_p] * 6 + [C.POINTER(C.c_double), C.POINTER(C.c_int),
                                                          C.POINTER(C.c_double), C.c_void_p]
    f.restype = C.c_int
    return f


@pytest.mark.parametrize("case", ["ot_rusanov", "rotor_hlle", "kh_hlld_rect"])
def test_noalloc_matches_handle_path_on_two_calls(case):
    import torch
    G = require_gpu()
    step = _noalloc(G)
    if case == "ot_rusanov":
        cfg, st = P.orszag_tang(64, riemann=RUSANOV)
    elif case == "rotor_hlle":
        cfg, st = P.rotor(72, riemann=HLLE)
    else:
        cfg, st = P.kelvin_helmholtz(48, riemann=HLLD)
    ref = G.Solver(cfg)
    ref.set_state(st)
    dev = [torch.from_numpy(a.copy()).cuda() for a in st]
    t = C.c_double(0.0)
    oc = C.c_int(1)
    dtn = C.c_double(0.0)
    ccfg = G.to_ccfg(cfg)
    torch.cuda.synchronize()
    for call in range(2):
        rc = step(C.byref(ccfg), *[C.c_void_p(x.data_ptr()) for x in dev], C.byref(t), C.byref(oc),
                  C.byref(dtn), None)
        assert rc == 0, G.lib().chimera_strerror(rc)
        ref.step(1)
        want = ref.get_state()
        d = ref.diag()
        for q in range(6):
            got = dev[q].cpu().numpy()
            assert np.array_equal(got, want[q]), (case, call, q)
        assert t.value == d["t"] and oc.value == d["output_count"] and dtn.value == d["dt"]
    ref.close()


def test_noalloc_rejects_oversize_and_bad_args():
    import torch
    G = require_gpu()
    step = _noalloc(G)
    big = G.to_ccfg(P.orszag_tang(8)[0].replace(nx=257, ny=256))
    x = torch.zeros(8, dtype=torch.float64, device="cuda")
    t, oc = C.c_double(0.0), C.c_int(1)
    ptr = C.c_void_p(x.data_ptr())
    assert step(C.byref(big), *([ptr] * 6), C.byref(t), C.byref(oc), None, None) == -8
    fp32 = G.to_ccfg(P.orszag_tang(8)[0].replace(precision=1))
    assert step(C.byref(fp32), *([ptr] * 6), C.byref(t), C.byref(oc), None, None) == -5
    assert step(None, *([ptr] * 6), C.byref(t), C.byref(oc), None, None) == -1


def test_noalloc_two_host_threads_are_serialised():
    """Two host threads, each on its own CUDA stream, step their own grids
    through the one scratch array at the same time: each must get the handle
    path's bits.  Both grids have one shape (different states), so every
    access stays inside the arrays whatever the interleaving."""
    import threading

    import torch
    G = require_gpu()
    step = _noalloc(G)
    cfg, st0 = P.rotor(64, riemann=HLLE)
    h = G.Solver(cfg)
    h.set_state(st0)
    h.step(1)
    st1 = h.get_state()
    h.close()
    states, wants = [st0, st1], []
    for st in states:
        r = G.Solver(cfg)
        r.set_state(st)
        outs = []
        for _ in range(4):
            r.step(1)
            outs.append(r.get_state())
        wants.append(outs)
        r.close()
    ccfg = G.to_ccfg(cfg)
    results, errors = [None, None], []
    start = threading.Barrier(2)

    def worker(k):
        try:
            s = torch.cuda.Stream()
            dev = [torch.from_numpy(a.copy()).cuda() for a in states[k]]
            torch.cuda.synchronize()
            t, oc, dtn = C.c_double(0.0), C.c_int(1), C.c_double(0.0)
            got = []
            start.wait(timeout=60)
            for _ in range(4):
                rc = step(C.byref(ccfg), *[C.c_void_p(x.data_ptr()) for x in dev], C.byref(t), C.byref(oc),
                          C.byref(dtn), C.c_void_p(s.cuda_stream))
                if rc:
                    errors.append((k, rc))
                    return
                got.append([x.cpu().numpy() for x in dev])
            results[k] = got
        except Exception as e:   # reported below, on the main thread
            errors.append((k, e))

    threads = [threading.Thread(target=worker, args=(k,)) for k in range(2)]
    for th in threads:
        th.start()
    for th in threads:
        th.join(timeout=120)
    assert not errors, errors
    for k in range(2):
        assert results[k] is not None
        for call in range(4):
            for q in range(6):
                assert np.array_equal(results[k][call][q], wants[k][call][q]), (k, call, q)


def test_noalloc_at_t_end_leaves_everything_untouched():
    """A call with t >= t_end takes no step (the reference's loop has ended):
    the six arrays, t, output_count and dt_next must come back bit for bit as
    they went in -- not the scratch's contents."""
    import torch
    G = require_gpu()
    step = _noalloc(G)
    cfg, st = P.rotor(64, riemann=HLLE)
    # run the scratch with another state first, so stale contents would show
    other = [torch.from_numpy(a.copy()).cuda() for a in P.orszag_tang(64)[1]]
    ocfg = G.to_ccfg(P.orszag_tang(64)[0])
    t0, oc0 = C.c_double(0.0), C.c_int(1)
    assert step(C.byref(ocfg), *[C.c_void_p(x.data_ptr()) for x in other], C.byref(t0), C.byref(oc0),
                None, None) == 0
    ccfg = G.to_ccfg(cfg)
    for t_start in (cfg.t_end, cfg.t_end + 0.25):
        dev = [torch.from_numpy(a.copy()).cuda() for a in st]
        torch.cuda.synchronize()
        t, oc, dtn = C.c_double(t_start), C.c_int(3), C.c_double(-7.5)
        rc = step(C.byref(ccfg), *[C.c_void_p(x.data_ptr()) for x in dev], C.byref(t), C.byref(oc),
                  C.byref(dtn), None)
        assert rc == 0, G.lib().chimera_strerror(rc)
        for q in range(6):
            assert np.array_equal(dev[q].cpu().numpy(), st[q]), q
        assert t.value == t_start and oc.value == 3 and dtn.value == -7.5


def test_noalloc_rejects_nonpositive_t_end():
    import torch
    G = require_gpu()
    step = _noalloc(G)
    cfg, st = P.orszag_tang(16)
    dev = [torch.from_numpy(a.copy()).cuda() for a in st]
    torch.cuda.synchronize()
    for t_end in (0.0, -1.0):
        bad = G.to_ccfg(cfg.replace(t_end=t_end))
        t, oc = C.c_double(0.0), C.c_int(1)
        assert step(C.byref(bad), *[C.c_void_p(x.data_ptr()) for x in dev], C.byref(t), C.byref(oc),
                    None, None) == -1
    for q in range(6):
        assert np.array_equal(dev[q].cpu().numpy(), st[q]), q


def test_noalloc_step_clipped_by_output_time():
    """A step that starts just before an output time: the dt is clipped to it
    (src/main.f90:82-83) and output_count advances.  State, t, output_count
    and the next dt equal the handle path's after chimera_set_time."""
    import torch
    G = require_gpu()
    step = _noalloc(G)
    cfg, st = P.orszag_tang(64, riemann=RUSANOV)
    cfg = cfg.replace(t_out=0.05, t_end=0.5)
    ccfg = G.to_ccfg(cfg)
    t_start = 0.05 - 1.0e-4       # well inside one CFL step of the output time
    ref = G.Solver(cfg)
    ref.set_state(st)
    ref.set_time(t_start, 1)
    dev = [torch.from_numpy(a.copy()).cuda() for a in st]
    torch.cuda.synchronize()
    t, oc, dtn = C.c_double(t_start), C.c_int(1), C.c_double(0.0)
    for call in range(2):
        rc = step(C.byref(ccfg), *[C.c_void_p(x.data_ptr()) for x in dev], C.byref(t), C.byref(oc),
                  C.byref(dtn), None)
        assert rc == 0, G.lib().chimera_strerror(rc)
        ref.step(1)
        want = ref.get_state()
        d = ref.diag()
        for q in range(6):
            assert np.array_equal(dev[q].cpu().numpy(), want[q]), (call, q)
        assert t.value == d["t"] and oc.value == d["output_count"] and dtn.value == d["dt"]
    assert oc.value == 2 and t.value > 0.05   # the first call landed on the output time
    ref.close()
