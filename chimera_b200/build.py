"""Build recipe for the CUDA library (``libchimera_gpu.so``, sm_100a).

nvcc compiles each translation unit for ``-gencode arch=compute_100a,code=sm_100a``
and links them into one shared library with a plain C-ABI
(``include/chimera_gpu.h``).  The FP64 unit is compiled with ``--fmad=false``
so no multiply-add is contracted (bit-compatible rounding with the reference
expressions).  Objects are cached by a hash of the sources and flags.
"""
from __future__ import annotations

import hashlib
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libchimera_gpu.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I" + CSRC, "-I" + INCLUDE]
UNITS = {
    "kernels_fp64.cu": ["--fmad=false"],
    "kernels_fp32.cu": ["-use_fast_math"],
    "chimera_api.cu": [],
    "noalloc.cu": ["--fmad=false"],
    "adjoint.cu": ["--fmad=false"],
    "unit_ops.cu": ["--fmad=false"],
}


def _nvcc():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _headers_digest():
    h = hashlib.sha256()
    for d in (CSRC, INCLUDE):
        for name in sorted(os.listdir(d)):
            if name.endswith((".h", ".cuh")):
                with open(os.path.join(d, name), "rb") as f:
                    h.update(name.encode() + f.read())
    return h.hexdigest()


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    hdr = _headers_digest()
    objs, jobs = [], []
    for unit, flags in UNITS.items():
        src = os.path.join(CSRC, unit)
        with open(src, "rb") as f:
            key = hashlib.sha256(f.read() + hdr.encode() + " ".join(ARCH + COMMON + flags).encode()).hexdigest()[:16]
        obj = os.path.join(BUILD, f"{unit}.{key}.o")
        if not os.path.exists(obj) or ptxas_info:
            cmd = [nvcc] + ARCH + COMMON + flags + (["-Xptxas", "-v"] if ptxas_info else []) + ["-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
            jobs.append((unit, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)))
        objs.append(obj)
    for unit, proc in jobs:   # the units compile in parallel
        _, err = proc.communicate()
        if proc.returncode != 0:
            raise RuntimeError(f"nvcc failed for {unit}:\n{err}")
        if ptxas_info:
            sys.stderr.write(err)
    cmd = [nvcc] + ARCH + ["-shared", "-o", LIB + ".tmp"] + objs + ["-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr}")
    os.replace(LIB + ".tmp", LIB)
    # objects of earlier source versions are never linked again: drop them
    current = {os.path.basename(o) for o in objs}
    for name in os.listdir(BUILD):
        if name.endswith(".o") and name not in current:
            os.remove(os.path.join(BUILD, name))
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, ptxas_info="-v" in sys.argv))
