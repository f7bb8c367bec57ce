"""Every kernel of the library is defined in exactly one translation unit.

The units are compiled with different floating-point flags (the FP64 units
without multiply-add contraction, the FP32 unit with fast math).  A kernel
template instantiated in two units is two device bodies under one symbol, and
a launch runs whichever module the runtime resolved the name to -- a bug that
showed as a one-ulp dt difference in some processes only.  This checks the
built objects' symbol tables (nm), with no GPU.
"""
import glob
import os
import shutil
import subprocess
from collections import defaultdict

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BUILD = os.path.join(ROOT, "chimera_b200", "_build")


def test_no_kernel_symbol_defined_in_two_units():
    objs = sorted(glob.glob(os.path.join(BUILD, "*.o")))
    if not objs or not shutil.which("nm"):
        pytest.skip("library objects not built here, or no nm")
    where = defaultdict(set)
    for obj in objs:
        out = subprocess.run(["nm", "-C", "--defined-only", obj], capture_output=True, text=True, check=True).stdout
        for line in out.splitlines():
            parts = line.split(None, 2)
            if len(parts) == 3 and parts[1] in ("T", "W", "t", "w") and "(chimera::StageArgs)" in parts[2]:
                where[parts[2]].add(os.path.basename(obj).split(".")[0])
    assert where, "no kernel symbols found"
    dups = {sym: units for sym, units in where.items() if len(units) > 1}
    assert not dups, dups
