"""The committed Athena++ Orszag-Tang fixture (tests/golden/ot_athena_t05.npz)
against its source: where the reference checkout is present, the hand-written
HDF5 reader reads the SHA-256-pinned file and reproduces the fixture."""
import hashlib
import os

import numpy as np
import pytest

from tests.golden import make_ot_athena as M

SRC = M.default_src()   # the fixture's source file, where CHIMERA_REFERENCE_DIR names the reference checkout


def test_fixture_shapes():
    z = np.load(M.OUT)
    assert float(z["sim_time"][0]) == 0.5
    for f in ("rho", "P"):
        for n in M.GRIDS:
            a = z[f"{f}_{n}"]
            assert a.shape == (n, n) and np.all(a > 0)


@pytest.mark.skipif(not SRC or not os.path.exists(SRC),
                    reason="CHIMERA_REFERENCE_DIR does not name a reference checkout")
def test_fixture_reproduced_from_pinned_file():
    with open(SRC, "rb") as f:
        assert hashlib.sha256(f.read()).hexdigest() == M.PINNED_SHA256
    from tests.golden.h5read import read_h5
    d = read_h5(SRC)
    assert set(d) >= {"rho/SNAPSHOT1", "P/SNAPSHOT1", "time/sim_time", "parameters/gamma"}
    z = np.load(M.OUT)
    for f in ("rho", "P"):
        assert np.array_equal(M.interp_to_grid(d[f"{f}/SNAPSHOT1"], 64).astype(np.float32), z[f"{f}_64"])
