"""Generate tests/golden/ot_athena_t05.npz from the reference's Athena++
Orszag-Tang solution (tests/validation/ot_reference.h5 of the reference:
500 x 500, t = 0.5, pinned there by SHA-256, test_validation.py:47).

The density and thermal pressure are interpolated bilinearly onto the
cell-centred N x N grids N = 64, 128, 256, exactly as the reference test's
_interp_to_grid does (test_validation.py:112-131), and stored as float32 (the
file's values are single-precision data).  Run in an environment that has the
reference checkout:

    python tests/golden/make_ot_athena.py path/to/ot_reference.h5

or with CHIMERA_REFERENCE_DIR set to the root of the reference checkout (the
file is then $CHIMERA_REFERENCE_DIR/tests/validation/ot_reference.h5).
"""
import hashlib
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
from tests.golden.h5read import read_h5  # noqa: E402

PINNED_SHA256 = "45e66217f6a81bae0831f8201b0cf6b10cdd75df3b5ecfd24c1e7899b5e92b5d"

def default_src():
    """The pinned file inside the reference checkout named by
    CHIMERA_REFERENCE_DIR, or None where that variable is unset."""
    root = os.environ.get("CHIMERA_REFERENCE_DIR")
    return os.path.join(root, "tests", "validation", "ot_reference.h5") if root else None

GRIDS = (64, 128, 256)
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ot_athena_t05.npz")


def interp_to_grid(arr, n_dst):
    """Bilinear interpolation of a square cell-centred array on [0,1]^2 onto
    an n_dst x n_dst cell-centred grid (np.interp along rows, then columns)."""
    n_src = arr.shape[0]
    x_src = (np.arange(n_src) + 0.5) / n_src
    x_dst = (np.arange(n_dst) + 0.5) / n_dst
    tmp = np.empty((n_src, n_dst))
    for i in range(n_src):
        tmp[i] = np.interp(x_dst, x_src, arr[i])
    out = np.empty((n_dst, n_dst))
    for j in range(n_dst):
        out[:, j] = np.interp(x_dst, x_src, tmp[:, j])
    return out


def main(path):
    with open(path, "rb") as f:
        digest = hashlib.sha256(f.read()).hexdigest()
    if digest != PINNED_SHA256:
        raise SystemExit(f"{path}: SHA-256 {digest} is not the pinned reference file")
    d = read_h5(path)
    t = float(d["time/sim_time"][0])
    assert abs(t - 0.5) < 1e-12, t
    arrays = {"sim_time": np.array([t]), "gamma": d["parameters/gamma"]}
    for field in ("rho", "P"):
        src = d[f"{field}/SNAPSHOT1"]
        assert src.shape == (500, 500)
        for n in GRIDS:
            arrays[f"{field}_{n}"] = interp_to_grid(src, n).astype(np.float32)
    np.savez_compressed(OUT, **arrays)
    print(f"wrote {OUT}: {sorted(arrays)}")


if __name__ == "__main__":
    src = sys.argv[1] if len(sys.argv) > 1 else default_src()
    if not src:
        raise SystemExit("usage: make_ot_athena.py path/to/ot_reference.h5 (or set CHIMERA_REFERENCE_DIR)")
    main(src)
