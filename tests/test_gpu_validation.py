"""The reference's quantitative Orszag-Tang validation
(tests/validation/test_validation.py) on the GPU backend, FP64, the
reference's default switches (Rusanov + MC + MOOD), snapshot at t = 0.5:

* tier 1: max / min of rho and thermal P at N = 128 inside the published
  ranges (Stone et al. 2008, Gardiner & Stone 2005) that the reference test
  uses (test_validation.py:36-39);
* tier 2: self-convergence -- N = 256 block-averaged to 64 and 128 as the
  surrogate truth; the L2 error must fall as N doubles with rate > 1
  (test_validation.py:239-279) -- and convergence toward the Athena++ 500^2
  solution the reference pins (tests/golden/ot_athena_t05.npz).
"""
import os

import numpy as np
import pytest

from chimera_b200 import problems as P
from chimera_b200.config import FP64
from tests.gpu_util import require_gpu

pytestmark = pytest.mark.gpu

RHO_MAX_BOUNDS = (0.42, 0.65)
RHO_MIN_BOUNDS = (0.03, 0.12)
P_MAX_BOUNDS = (0.38, 0.72)
P_MIN_BOUNDS = (0.008, 0.07)


@pytest.fixture(scope="module")
def ot_half():
    """rho and thermal P at t = 0.5 for N = 64, 128, 256."""
    require_gpu()
    from chimera_b200 import run
    out = {}
    for n in (64, 128, 256):
        cfg, st = P.orszag_tang(n, t_end=0.5)
        snaps = run.run(cfg, st, FP64)
        snap = min(snaps, key=lambda s: abs(s["t"] - 0.5))
        assert abs(snap["t"] - 0.5) < 1e-9
        out[n] = snap
    return out


def test_ot128_published_bounds(ot_half):
    rho, p = ot_half[128]["rho"], ot_half[128]["P"]
    print(f"OT N=128 t=0.5: rho [{rho.min():.4f}, {rho.max():.4f}]  P [{p.min():.4f}, {p.max():.4f}]")
    assert RHO_MAX_BOUNDS[0] < rho.max() < RHO_MAX_BOUNDS[1]
    assert RHO_MIN_BOUNDS[0] < rho.min() < RHO_MIN_BOUNDS[1]
    assert P_MAX_BOUNDS[0] < p.max() < P_MAX_BOUNDS[1]
    assert P_MIN_BOUNDS[0] < p.min() < P_MIN_BOUNDS[1]


def _coarsen(a, f):
    m = a.shape[0] // f
    return a.reshape(m, f, m, f).mean(axis=(1, 3))


def _l2(a, b):
    return float(np.sqrt(np.mean((a - b) ** 2)))


@pytest.mark.parametrize("field", ["rho", "P"])
def test_ot_self_convergence(ot_half, field):
    ref = ot_half[256][field]
    e64 = _l2(ot_half[64][field], _coarsen(ref, 4))
    e128 = _l2(ot_half[128][field], _coarsen(ref, 2))
    rate = np.log2(e64 / e128)
    print(f"OT {field}: L2(64) = {e64:.3e}, L2(128) = {e128:.3e}, rate {rate:.2f}")
    assert e128 < e64 and rate > 1.0


@pytest.mark.parametrize("field", ["rho", "P"])
def test_ot_converges_toward_athena(ot_half, field):
    """Part 2 of the reference's convergence test (test_validation.py:291-307):
    the L2 error against the Athena++ 500^2 solution (bilinearly interpolated
    to each grid; tests/golden/make_ot_athena.py) falls as N doubles."""
    z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ot_athena_t05.npz"))
    errs = {n: _l2(ot_half[n][field], z[f"{field}_{n}"].astype(np.float64)) for n in (64, 128, 256)}
    print(f"OT {field} vs Athena++: " + ", ".join(f"N={n}: {e:.3e}" for n, e in errs.items()))
    assert errs[128] < errs[64] and errs[256] < errs[128]
