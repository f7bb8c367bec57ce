"""The reference's stress suite (tests/stress/test_stress.py:76-234) on the CPU
oracle: GRF members of 64^2 (seeds 42 and 43 at the default draw, a target
sonic Mach number of 5 before the speed cap, a target plasma beta of 0.1) run
to t = 0.05 with the reference's tOut = 0.01, i.e. to the fifth snapshot.
Every snapshot must have finite, positive density and thermal pressure, the
total mass must stay put, and the realised Mach number and beta must be in
the ranges the reference checks.  The GPU path is bit-identical to the oracle
in FP64 (tests/test_gpu_parity.py), so these hold for it too."""
import numpy as np
import pytest

from chimera_b200 import problems as P
from chimera_b200 import run
from tests.snapshots import mass_drift, oracle_snapshots

N, SEED = 64, 42                           # tests/stress/test_stress.py GRF_N, GRF_SEED
M_S_BOUNDS, BETA_BOUNDS = (0.01, 20.0), (0.01, 100.0)


def _member(**kw):
    cfg, st = P.grf_member(N, kw.pop("seed", SEED), **kw)
    return cfg.replace(t_end=0.05, t_out=0.01), st


def _realised(cfg, st):
    """Sonic Mach number and plasma beta of the initial state, as the
    reference stores them (run.initial_parameters)."""
    p = run.initial_parameters(cfg, st, 5)
    return p["M_s"], p["beta"]


def _check_run(oracle, cfg, st):
    snaps = oracle_snapshots(oracle, cfg, st)
    assert len(snaps) >= 5, len(snaps)
    for s in snaps:
        for f in ("rho", "P", "Vx", "Vy", "Bx", "By"):
            assert np.all(np.isfinite(s[f])), f
        assert s["rho"].min() > 0.0
        assert s["P"].min() > 0.0
    assert mass_drift(snaps) < 1e-10
    return snaps


@pytest.mark.parametrize("seed", [SEED, SEED + 1])
def test_grf_completes_positive_and_plausible(oracle, seed):
    cfg, st = _member(seed=seed)
    mach, beta = _realised(cfg, st)
    assert cfg.gamma > 1.0
    assert M_S_BOUNDS[0] < mach < M_S_BOUNDS[1]
    assert BETA_BOUNDS[0] < beta < BETA_BOUNDS[1]
    _check_run(oracle, cfg, st)


def test_high_mach_stable(oracle):
    """Target M_s = 5: the cap step scales the velocities down by
    3 / max(c_f + |v|), so the run starts on the cap's path with steep
    velocity gradients."""
    cfg, st = _member(mach=5.0)
    _, uncapped = P.grf_member(N, SEED, mach=5.0, cf_cap=1e30)
    assert not np.array_equal(st[1], uncapped[1])        # the cap rescaled the momenta
    mach, _ = _realised(cfg, st)
    assert M_S_BOUNDS[0] < mach < 5.0
    _check_run(oracle, cfg, st)


def test_low_beta_stable(oracle):
    """Target beta = 0.1: thermal pressure is a small residual of the total
    energy, the regime of the proportional pressure floor; the realised beta
    is magnetically dominated (< 0.5)."""
    cfg, st = _member(beta=0.1)
    _, beta = _realised(cfg, st)
    assert beta < 0.5
    _check_run(oracle, cfg, st)
