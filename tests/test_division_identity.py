"""Evidence for an FP64 division through a shared, correctly rounded
reciprocal plus one Markstein correction step: it must reproduce IEEE
division bit for bit on random quotients (tests/numerics/div_sweep.c).  The
default sweep is 1.6e7 quotients; CHIMERA_DIV_SWEEP_SCALE=100 runs 1.6e9."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def test_shared_reciprocal_division_matches_ieee(tmp_path):
    cc = shutil.which("gcc")
    if cc is None:
        pytest.skip("no host compiler")
    exe = tmp_path / "div_sweep"
    subprocess.run([cc, "-O2", "-ffp-contract=off", "-o", str(exe), os.path.join(HERE, "numerics", "div_sweep.c"),
                    "-lm"], check=True)
    scale = int(os.environ.get("CHIMERA_DIV_SWEEP_SCALE", "1"))
    out = subprocess.run([str(exe), str(1000000 * scale), "100", str(100000 * scale)], capture_output=True,
                         text=True, check=True, timeout=3600).stdout.split()
    total, bad = int(out[0]), int(out[1])
    assert total == 16000000 * scale and bad == 0
