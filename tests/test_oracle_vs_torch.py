"""The two independent FP64 restatements (C, oracle/chimera_oracle.c, and
PyTorch, oracle/torch_ref.py) must agree bit for bit on every switch
combination, boundary mix and rectangular grids."""
import numpy as np
import pytest
import torch

from chimera_b200 import problems as P
from chimera_b200.config import HLLD, HLLE, VAN_LEER, BC_OUTFLOW, BC_PERIODIC
from oracle import torch_ref as T

CASES = {
    "ot_rusanov_mc": lambda: P.orszag_tang(24),
    "ot_hlle": lambda: P.orszag_tang(24, riemann=HLLE),
    "ot_hlld_vl": lambda: P.orszag_tang(24, riemann=HLLD, limiter=VAN_LEER),
    "rotor_hlle": lambda: P.rotor(40),
    "rotor_hlld_nomood": lambda: P.rotor(40, riemann=HLLD, mood=False),
    "field_loop_rect": lambda: P.field_loop(32, 16),
    "kh_rect_hlld": lambda: P.kelvin_helmholtz(24, riemann=HLLD),
    "grf": lambda: P.grf_member(24, 7),
    "mixed_bc": lambda: _mixed(),
    "no_slope_limiting": lambda: _nolim(),
}


def _mixed():
    cfg, st = P.orszag_tang(24)
    return cfg.replace(bc=(BC_PERIODIC, BC_PERIODIC, BC_OUTFLOW, BC_OUTFLOW)), st


def _nolim():
    cfg, st = P.orszag_tang(24)
    return cfg.replace(slope_limiting=False), st


@pytest.mark.parametrize("case", sorted(CASES))
def test_c_and_torch_agree_bitwise(oracle, case):
    cfg, st = CASES[case]()
    s = oracle.State(st)
    dts = oracle.run(cfg, s, 12)
    U = [torch.from_numpy(a.copy()) for a in st]
    t, oc = 0.0, 1
    for k in range(12):
        dt = T.cfl_dt(cfg, U, t, oc)
        assert dt == dts[k]
        U = T.rk3_step(cfg, U, dt)
        t += dt
        if t >= oc * cfg.t_out or t >= cfg.t_end:
            oc += 1
    for q in range(6):
        assert np.array_equal(U[q].numpy(), s.a[q]), q
