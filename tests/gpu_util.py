"""Helpers shared by the GPU tests: load the CUDA library (failing loudly if it
is missing -- there is no CPU fallback) and run the oracle beside it."""
import numpy as np
import pytest


def require_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test collected without a CUDA device")
    from chimera_b200 import build, gpu
    import os
    if not os.path.exists(gpu.LIB_PATH):
        build.build()
    gpu.lib()
    return gpu


def l1_rel(a, b):
    """L1 relative error of a against reference b (per field)."""
    den = np.sum(np.abs(b))
    return float(np.sum(np.abs(a - b)) / den) if den > 0 else float(np.sum(np.abs(a - b)))


def max_ulp(a, b):
    ai = a.view(np.int64)
    bi = b.view(np.int64)
    ai = np.where(ai < 0, np.int64(-(2 ** 63)) - ai, ai)
    bi = np.where(bi < 0, np.int64(-(2 ** 63)) - bi, bi)
    return int(np.max(np.abs(ai - bi))) if a.size else 0
