"""The reference's quantitative Orszag-Tang validation
(tests/validation/test_validation.py) on the CPU oracle, with the reference's
default switches (Rusanov + MC + MOOD), state at t = 0.5:

* tier 1: max / min of rho and thermal P at N = 128 inside the published
  ranges (Stone et al. 2008, Gardiner & Stone 2005) the reference test uses
  (test_validation.py:36-39);
* convergence toward the Athena++ 500^2 solution the reference pins
  (tests/golden/ot_athena_t05.npz, bilinearly interpolated to each grid): the
  L2 error falls from N = 64 to N = 128 (test_validation.py:291-307).

The GPU form (tests/test_gpu_validation.py) adds N = 256 and the
self-convergence rate; the FP64 GPU path is bit-identical to the oracle."""
import os

import numpy as np
import pytest

from chimera_b200 import problems as P

RHO_MAX_BOUNDS = (0.42, 0.65)
RHO_MIN_BOUNDS = (0.03, 0.12)
P_MAX_BOUNDS = (0.38, 0.72)
P_MIN_BOUNDS = (0.008, 0.07)


@pytest.fixture(scope="module")
def ot_half(oracle):
    """rho and thermal P at t = 0.5 for N = 64 and 128."""
    out = {}
    for n in (64, 128):
        cfg, st = P.orszag_tang(n, t_end=0.5)
        s = oracle.State(st)
        oracle.run(cfg, s, 100000)
        assert s.t == 0.5
        rho, _, _, Ptot, Bx, By = oracle.primitives(cfg, s.a)
        out[n] = {"rho": rho, "P": Ptot - 0.5 * (Bx * Bx + By * By)}
    return out


def test_ot128_published_bounds(ot_half):
    rho, p = ot_half[128]["rho"], ot_half[128]["P"]
    assert RHO_MAX_BOUNDS[0] < rho.max() < RHO_MAX_BOUNDS[1]
    assert RHO_MIN_BOUNDS[0] < rho.min() < RHO_MIN_BOUNDS[1]
    assert P_MAX_BOUNDS[0] < p.max() < P_MAX_BOUNDS[1]
    assert P_MIN_BOUNDS[0] < p.min() < P_MIN_BOUNDS[1]


@pytest.mark.parametrize("field", ["rho", "P"])
def test_ot_converges_toward_athena(ot_half, field):
    z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ot_athena_t05.npz"))
    err = {n: float(np.sqrt(np.mean((ot_half[n][field] - z[f"{field}_{n}"].astype(np.float64)) ** 2)))
           for n in (64, 128)}
    assert err[128] < err[64], err
