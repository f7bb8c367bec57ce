"""The reference's structural suite (tests/structural/test_structural.py:18-119)
on CPU: the Orszag-Tang vortex at N = 32 with the reference's tEnd = 1.0 and
tOut = 0.01, advanced by the oracle, its snapshots written by
``run.write_snapshots`` (the writer ``run_sim`` uses, with the HDF5 paths of
src/mhd_write_h5.f90:13-194 as archive keys) and read back by
``run.read_snapshots``.  The same checks on a GPU run are in
tests/test_gpu_properties.py."""
import numpy as np
import pytest

from chimera_b200 import run
from tests.snapshots import oracle_snapshots

N = 32
FIELDS = ("rho", "P", "Bx", "By", "Vx", "Vy")
PARAMS = ("parameters/gamma", "parameters/M_s", "parameters/beta")


def _keys(data, field):
    return sorted((k for k in data if k.startswith(field + "/")), key=lambda k: int(k.split("SNAPSHOT")[1]))


@pytest.fixture(scope="module")
def data(oracle, tmp_path_factory):
    cfg, st, params = run.reference_problem(1, N)
    snaps = oracle_snapshots(oracle, cfg, st)
    path = run.write_snapshots(str(tmp_path_factory.mktemp("snap") / f"test_p1_N{N}_s0"), snaps, params)
    assert path.endswith(".npz")
    return run.read_snapshots(path)


def test_all_fields_time_and_parameters_present(data):
    for f in FIELDS:
        assert f + "/SNAPSHOT1" in data, f
    assert "time/sim_time" in data
    for p in PARAMS:
        assert p in data and data[p].shape == (1,), p
    assert data["parameters/gamma"][0] > 1.0


def test_snapshot_shapes_and_counts(data):
    counts = {f: len(_keys(data, f)) for f in FIELDS}
    assert len(set(counts.values())) == 1, counts
    n = counts["rho"]
    assert n >= 5
    assert data["time/sim_time"].shape == (n,)
    for f in FIELDS:
        for k in _keys(data, f):
            assert data[k].shape == (N, N), k


def test_times_monotonically_increasing(data):
    t = data["time/sim_time"]
    assert np.all(np.diff(t) > 0)
    assert abs(t[0] - 0.01) < 1e-12 and abs(t[-1] - 1.0) < 1e-12   # tOut clipping (src/main.f90:82-83)


def test_p_dataset_is_thermal_pressure(data):
    """Orszag-Tang starts at uniform thermal pressure 5/(12 pi) ~ 0.133 and
    mean magnetic pressure 1/(8 pi) ~ 0.040: a first-snapshot mean below 0.16
    separates thermal from total pressure."""
    keys = _keys(data, "P")
    first, last = data[keys[0]], data[keys[-1]]
    assert first.min() > 0.0 and last.min() > 0.0
    assert first.mean() < 0.16
    assert abs(first.mean() - 5.0 / (12.0 * np.pi)) < 0.01
