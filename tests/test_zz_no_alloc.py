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
