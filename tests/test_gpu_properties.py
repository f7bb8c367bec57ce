"""The reference's physics property suites (tests/physics/test_physics.py,
tests/physics/test_rk3.py) re-pointed at the GPU backend: whole runs made by
chimera_b200.run (the reference's problem set-ups, time loop and snapshot
cadence, tEnd = 1.0 / 0.5 as in the oracle suites), in the plain FP64 form and
in the FP32-bulk form, plus the snapshot archive's layout
(tests/structural/test_structural.py) and its agreement with the oracle."""
import numpy as np
import pytest

from chimera_b200 import problems as P
from chimera_b200.config import FP32_BULK, FP64, MC, RUSANOV
from tests.gpu_util import require_gpu
from tests.snapshots import energy_mean, field_loop_l1, mass_drift, oracle_snapshots

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def R():
    require_gpu()
    from chimera_b200 import run
    return run


def _ot(n, t_end):
    return P.orszag_tang(n, t_end=t_end)


def _fl(n):
    return P.field_loop(n, n, 1.0, 1.0, v=(-2.0, -1.0), riemann=RUSANOV, limiter=MC, t_end=1.0)


@pytest.fixture(scope="module", params=[FP64, FP32_BULK], ids=["fp64", "fp32"])
def runs(R, request):
    prec = request.param
    out = {"prec": prec}
    for key, (cfg, st) in {"ot32": _ot(32, 1.0), "ot64": _ot(64, 0.5), "fl32": _fl(32), "fl64": _fl(64)}.items():
        out[key] = (cfg, R.run(cfg, st, prec))
    return out


# mass conservation: 1e-10 in FP64 (tests/physics/test_physics.py:46-60); the
# FP32-bulk form stores the state in FP32, so its bound is FP32 roundoff
def _mass_tol(prec):
    return 1e-10 if prec == FP64 else 1e-6


def test_mass_conserved(runs):
    tol = _mass_tol(runs["prec"])
    assert mass_drift(runs["ot32"][1]) < tol
    assert mass_drift(runs["fl32"][1]) < tol


def test_positivity(runs):   # tests/physics/test_physics.py:66-84
    for key in ("ot32", "fl32", "ot64"):
        snaps = runs[key][1]
        assert min(s["rho"].min() for s in snaps) > 0.0
        assert min(s["P"].min() for s in snaps) > 0.0


def test_snapshot_cadence(runs):   # tests/physics/test_physics.py:89-92; one snapshot per tOut
    snaps = runs["ot32"][1]
    t = np.array([s["t"] for s in snaps])
    assert 99 <= len(snaps) <= 101 and np.all(np.diff(t) > 0) and t[-1] >= 1.0 - 1e-12
    assert np.all(np.abs(t[:99] - 0.01 * np.arange(1, 100)) < 1e-12)   # dt is clipped to each tOut


def test_field_loop_no_density_spike(runs):   # tests/physics/test_rk3.py:84-101
    snaps = runs["fl64"][1]
    rho0 = snaps[0]["rho"].max()
    assert max(s["rho"].max() for s in snaps) <= rho0 + 1e-3 * rho0


def test_ot_pressure_floor_fraction(runs):   # tests/physics/test_rk3.py:103-134
    snaps = runs["ot64"][1]
    assert max(float(np.sum(s["P"] <= 1e-11)) / s["P"].size for s in snaps) < 1e-3


def test_ot_energy(runs):   # tests/physics/test_rk3.py:151-186
    cfg, snaps = runs["ot64"]
    t = np.array([s["t"] for s in snaps])
    E = np.array([energy_mean(s, cfg.gamma) for s in snaps])
    idx = int(np.argmin(np.abs(t - 0.5)))
    assert abs(t[idx] - 0.5) <= 0.02 and abs((E[idx] - E[0]) / E[0]) < 0.03
    early = E[t <= 0.2]
    # energy may not grow before t = 0.2: 1e-6 relative in FP64; FP32 storage
    # rounding of the 4096 cells' energies allows 1e-6 per step more
    tol = 1e-6 if runs["prec"] == FP64 else 1e-5
    assert len(early) >= 2 and max(0.0, float(np.max(np.diff(early)))) < tol * abs(E[0])


def test_field_loop_convergence(runs):   # tests/physics/test_physics.py:118-141
    e32, e64 = field_loop_l1(runs["fl32"][1]), field_loop_l1(runs["fl64"][1])
    assert e64 < e32 and e32 / e64 >= 1.5


def test_fp64_snapshots_equal_the_oracle(R, oracle):
    """The FP64 run's snapshots are the oracle's, bit for bit (same steps,
    same output times, primitives from the same routines)."""
    cfg, st = _ot(32, 0.3)
    gpu_snaps = R.run(cfg, st, FP64)
    ref = oracle_snapshots(oracle, cfg, st)
    assert len(gpu_snaps) == len(ref) == 30
    for a, b in zip(gpu_snaps, ref):
        assert a["t"] == b["t"]
        for f in ("rho", "Vx", "Vy", "P", "Bx", "By"):
            assert np.array_equal(a[f], b[f]), f


@pytest.mark.parametrize("problem_type", [1, 2, 3, 4, 5])
def test_run_sim_archive_layout(R, tmp_path, problem_type):
    """The archive of every reference problem has the reference file's paths
    (tests/structural/test_structural.py): six groups of SNAPSHOT<k> arrays of
    shape (N, N), time/sim_time increasing, parameters/{gamma, M_s, beta}."""
    N = 32
    path = R.run_sim(problem_type, N, seed=3, out_dir=str(tmp_path), t_end=0.05)
    data = R.read_snapshots(path)
    keys = R.snapshot_keys(data)
    assert 5 <= len(keys) <= 6 and keys[0] == "SNAPSHOT1"
    for f in R.FIELDS:
        assert R.snapshot_keys(data, f) == keys
        for k in keys:
            arr = data[f"{f}/{k}"]
            assert arr.shape == (N, N)
            assert np.all(np.isfinite(arr))
    t = data["time/sim_time"]
    assert t.shape == (len(keys),) and np.all(np.diff(t) > 0) and abs(t[-1] - 0.05) < 1e-12
    for name in ("gamma", "M_s", "beta"):
        assert data[f"parameters/{name}"].shape == (1,)
    if problem_type == 5:
        assert data["parameters/M_s"][0] > 0 and data["parameters/beta"][0] > 0
