"""The reference's integral property checks (tests/physics/test_physics.py,
tests/physics/test_rk3.py), run on the CPU oracle with the reference's default
switches (Rusanov + MC + MOOD) and tEnd = 1.0."""
import numpy as np
import pytest

from chimera_b200 import problems as P
from tests.snapshots import energy_mean, field_loop_l1, mass_drift, oracle_snapshots


@pytest.fixture(scope="module")
def ot32(oracle):
    cfg, st = P.orszag_tang(32, t_end=1.0)
    return cfg, oracle_snapshots(oracle, cfg, st)


@pytest.fixture(scope="module")
def ot64(oracle):
    cfg, st = P.orszag_tang(64, t_end=0.5)
    return cfg, oracle_snapshots(oracle, cfg, st)


def _fl(oracle, n):
    # the reference field loop: unit square, v = (-2, -1) (src/mhd_init.f90:360-391)
    from chimera_b200.config import MC, RUSANOV
    cfg, st = P.field_loop(n, n, 1.0, 1.0, v=(-2.0, -1.0), riemann=RUSANOV, limiter=MC, t_end=1.0)
    return cfg, oracle_snapshots(oracle, cfg, st)


@pytest.fixture(scope="module")
def fl32(oracle):
    return _fl(oracle, 32)


@pytest.fixture(scope="module")
def fl64(oracle):
    return _fl(oracle, 64)


# tests/physics/test_physics.py:46-60
def test_mass_conserved_ot(ot32):
    assert mass_drift(ot32[1]) < 1e-10


def test_mass_conserved_field_loop(fl32):
    assert mass_drift(fl32[1]) < 1e-10


# tests/physics/test_physics.py:66-84
def test_positivity_ot(ot32):
    assert min(s["rho"].min() for s in ot32[1]) > 0.0
    assert min(s["P"].min() for s in ot32[1]) > 0.0


def test_positivity_field_loop(fl32):
    assert min(s["rho"].min() for s in fl32[1]) > 0.0


# tests/physics/test_physics.py:89-92
def test_snapshot_count_ot(ot32):
    assert len(ot32[1]) >= 5
    t = [s["t"] for s in ot32[1]]
    assert all(b > a for a, b in zip(t, t[1:]))


# tests/physics/test_rk3.py:84-101
def test_field_loop_no_density_spike(fl64):
    rho0 = fl64[1][0]["rho"].max()
    hi = max(s["rho"].max() for s in fl64[1])
    assert hi <= rho0 + 1e-3 * rho0


# tests/physics/test_rk3.py:103-134
def test_ot_pressure_floor_fraction(ot64):
    frac = max(float(np.sum(s["P"] <= 1e-12 * 10)) / s["P"].size for s in ot64[1])
    assert frac < 1e-3


# tests/physics/test_rk3.py:151-186
def test_ot_energy_loss_half_period(ot64):
    cfg, snaps = ot64
    t = np.array([s["t"] for s in snaps])
    E = np.array([energy_mean(s, cfg.gamma) for s in snaps])
    idx = int(np.argmin(np.abs(t - 0.5)))
    assert abs(t[idx] - 0.5) <= 0.02
    assert abs((E[idx] - E[0]) / E[0]) < 0.03


def test_ot_energy_monotone_early(ot64):
    cfg, snaps = ot64
    t = np.array([s["t"] for s in snaps])
    E = np.array([energy_mean(s, cfg.gamma) for s in snaps])
    early = E[t <= 0.2]
    assert len(early) >= 2
    assert max(0.0, float(np.max(np.diff(early)))) < 1e-6 * abs(E[0])


# tests/physics/test_physics.py:118-141
def test_field_loop_convergence(fl32, fl64):
    e32, e64 = field_loop_l1(fl32[1]), field_loop_l1(fl64[1])
    assert e64 < e32
    assert e32 / e64 >= 1.5
