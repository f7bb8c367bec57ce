"""The FP64 division through a reciprocal fixed for the launch (div_by in
chimera_b200/csrc/mhd_device.cuh: one Markstein correction step inside its
exact range, IEEE division outside it) must reproduce IEEE division bit for
bit (tests/numerics/div_sweep.c mirrors it on the host): random quotients,
quotients within a few 2^-106 of a rounding midpoint, and the numerators at
the ends of the range.  The default sweep is about 2.4e7 quotients;
CHIMERA_DIV_SWEEP_SCALE=100 runs about 2.4e9."""
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
    out = subprocess.run([str(exe), str(1000000 * scale), "100", str(100000 * scale), str(4000000 * scale)],
                         capture_output=True, text=True, check=True, timeout=3600).stdout.split()
    total, bad = int(out[0]), int(out[1])
    # 13 fixed and 100 random denominators, most of the near-midpoint draws, the range ends
    assert total > 23000000 * scale and bad == 0
