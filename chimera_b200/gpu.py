"""Python binding of the CUDA drop-in (``include/chimera_gpu.h``) via ctypes.

This is how the Python run scripts reach the GPU path (the reference reaches
its solver only through ``subprocess`` + HDF5, ``scripts/run_mhd.py:197-202``).
Arrays are ``(ny, nx)`` float64 (x fastest, the Fortran ``(nx, ny)`` layout):
numpy arrays are passed as host memory, CUDA torch tensors as device memory.

There is no CPU fallback: if ``libchimera_gpu.so`` is missing or no CUDA
device is present, construction raises.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Sequence

import numpy as np

from .config import SolverConfig

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libchimera_gpu.so")

OK = 0
ERR = {
    -1: "CHIMERA_ERR_BAD_ARG", -2: "CHIMERA_ERR_CUDA", -3: "CHIMERA_ERR_NONFINITE",
    -4: "CHIMERA_ERR_TIMEOUT", -5: "CHIMERA_ERR_UNSUPPORTED", -6: "CHIMERA_ERR_NO_DEVICE",
    -7: "CHIMERA_ERR_NOMEM", -8: "CHIMERA_ERR_TOO_LARGE",
}
HOST, DEVICE = 0, 1


class ChimeraError(RuntimeError):
    def __init__(self, code: int, what: str):
        super().__init__(f"{what}: {ERR.get(code, code)} ({_strerror(code)})")
        self.code = code


class CCfg(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int),
        ("dx", C.c_double), ("dy", C.c_double), ("gamma", C.c_double),
        ("courant", C.c_double), ("t_out", C.c_double), ("t_end", C.c_double),
        ("bc_xlo", C.c_int), ("bc_xhi", C.c_int), ("bc_ylo", C.c_int), ("bc_yhi", C.c_int),
        ("riemann", C.c_int), ("limiter", C.c_int), ("use_slope_limiting", C.c_int),
        ("mood", C.c_int), ("precision", C.c_int),
    ]


class CDiag(C.Structure):
    _fields_ = [
        ("t", C.c_double), ("dt", C.c_double), ("output_count", C.c_int), ("active", C.c_int),
        ("steps", C.c_ulonglong), ("divb_max", C.c_double), ("divb_mean", C.c_double),
        ("bmax", C.c_double), ("divb_rel", C.c_double), ("mass", C.c_double),
        ("energy", C.c_double), ("cfl_speed", C.c_double), ("mood_resets", C.c_ulonglong),
        ("floor_hits", C.c_ulonglong), ("status", C.c_uint),
    ]


_lib = None


def lib():
    """Load the in-tree library (built by ``chimera_b200.build``)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run `python -m chimera_b200.build` "
                               "(there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        dp = C.POINTER(C.c_double)
        L.chimera_strerror.restype = C.c_char_p
        L.chimera_strerror.argtypes = [C.c_int]
        L.chimera_create.argtypes = [C.POINTER(CCfg), P, C.POINTER(P)]
        L.chimera_batch_create.argtypes = [C.c_int, C.POINTER(CCfg), P, C.POINTER(P)]
        L.chimera_destroy.argtypes = [P]
        L.chimera_destroy.restype = None
        io = [P, C.c_int, P, P, P, P, P, P, C.c_int, C.c_int]
        L.chimera_batch_set_state.argtypes = io
        L.chimera_batch_get_state.argtypes = io
        L.chimera_get_stage_buffer.argtypes = io
        L.chimera_batch_set_time.argtypes = [P, C.c_int, C.c_double, C.c_int]
        L.chimera_step.argtypes = [P, C.c_int]
        L.chimera_step_host.argtypes = [P, P * 6, P * 6, C.c_int]
        L.chimera_advance.argtypes = [P, C.c_int, C.POINTER(C.c_int)]
        L.chimera_advance_output.argtypes = [P, C.c_int, C.POINTER(C.c_int)]
        L.chimera_stage.argtypes = [P, C.c_int, C.c_double]
        L.chimera_batch_diag.argtypes = [P, C.c_int, C.POINTER(CDiag)]
        L.chimera_set_counters.argtypes = [P, C.c_int]
        L.chimera_set_graph_steps.argtypes = [P, C.c_int]
        L.chimera_set_profiling.argtypes = [P, C.c_int]
        L.chimera_get_profile.argtypes = [P, C.POINTER(C.c_double), C.POINTER(C.c_longlong), C.c_int]
        L.chimera_autotune.argtypes = [P, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double)]
        L.chimera_variant_count.argtypes = [P]
        L.chimera_set_variant.argtypes = [P, C.c_int]
        L.chimera_get_variant.argtypes = [P, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                          C.POINTER(C.c_int)]
        L.chimera_stream.argtypes = [P]
        L.chimera_stream.restype = P
        L.chimera_halo_pack.argtypes = [P, C.c_int, P, P]
        L.chimera_halo_unpack.argtypes = [P, C.c_int, P, P]
        L.chimera_slab_ghost_rows.argtypes = [P, C.c_int, C.c_int]
        L.chimera_refresh_dt.argtypes = [P, P]
        L.chimera_set_dt_device.argtypes = [P, P]
        L.chimera_get_dt_device.argtypes = [P, P]
        _lib = L
    return _lib


def _strerror(code: int) -> str:
    try:
        return lib().chimera_strerror(int(code)).decode()
    except Exception:  # pragma: no cover - library missing
        return "?"


def _check(rc: int, what: str) -> None:
    if rc != OK:
        raise ChimeraError(rc, what)


def to_ccfg(cfg: SolverConfig) -> CCfg:
    return CCfg(cfg.nx, cfg.ny, cfg.dx, cfg.dy, cfg.gamma, cfg.courant, cfg.t_out, cfg.t_end,
                cfg.bc[0], cfg.bc[1], cfg.bc[2], cfg.bc[3], cfg.riemann, cfg.limiter,
                int(bool(cfg.slope_limiting)), int(bool(cfg.mood)), int(getattr(cfg, "precision", 0)))


def _ptrs(arrays, nx, ny, out=False):
    """(pointers, ld, where, keepalive) for 6 arrays (numpy host or torch cuda).

    float64 arrays with unit x stride are passed as they are, with their row
    pitch as ld (views of padded arrays included).  Other numpy inputs are
    converted to a dense copy; an output (``out``) that would need a copy is
    rejected, since the result would land in the copy."""
    ptrs, keep = [], []
    where = None
    ld = nx
    for a in arrays:
        if hasattr(a, "data_ptr"):
            import torch
            if a.dtype != torch.float64:
                raise TypeError("tensors must be float64")
            if tuple(a.shape) != (ny, nx) or a.stride(1) != 1:
                raise ValueError(f"expected a ({ny}, {nx}) tensor with unit x stride")
            w = DEVICE if a.is_cuda else HOST
            ld_a, p = a.stride(0), a.data_ptr()
        else:
            direct = (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.ndim == 2 and a.shape == (ny, nx)
                      and a.strides[1] == 8 and a.strides[0] % 8 == 0 and a.strides[0] >= 8 * nx)
            if not direct:
                if out:
                    raise ValueError(f"output arrays must be ({ny}, {nx}) float64 with unit x stride")
                a = np.ascontiguousarray(a, dtype=np.float64)
                if a.shape != (ny, nx):
                    raise ValueError(f"expected shape ({ny}, {nx}), got {a.shape}")
            keep.append(a)
            w, ld_a, p = HOST, a.strides[0] // 8, a.ctypes.data
        if where is None:
            where, ld = w, ld_a
        elif w != where or ld_a != ld:
            raise ValueError("all six arrays must live in the same memory with the same pitch")
        ptrs.append(C.c_void_p(p))
    return ptrs, ld, where, keep


class Solver:
    """A batch of grids (one grid when given a single config) on the GPU."""

    def __init__(self, cfgs, stream: int | None = None):
        if isinstance(cfgs, SolverConfig):
            cfgs = [cfgs]
        self.cfgs: list[SolverConfig] = list(cfgs)
        arr = (CCfg * len(self.cfgs))(*[to_ccfg(c) for c in self.cfgs])
        h = C.c_void_p()
        _check(lib().chimera_batch_create(len(self.cfgs), arr, C.c_void_p(stream), C.byref(h)),
               "chimera_batch_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().chimera_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
        return False

    @property
    def handle(self):
        return self._h

    @property
    def stream(self) -> int:
        return lib().chimera_stream(self._h) or 0

    def set_state(self, arrays: Sequence, member: int = 0):
        """Six conserved fields (Mass, Momx, Momy, Energy, b_x, b_y) of member
        ``member`` in: numpy arrays or CPU tensors are read completely before
        the call returns (page-locked ones included); CUDA tensors are copied
        in order on the solver's stream."""
        c = self.cfgs[member]
        p, ld, where, keep = _ptrs(arrays, c.nx, c.ny)
        _check(lib().chimera_batch_set_state(self._h, member, *p, ld, where), "set_state")

    def get_state(self, member: int = 0, out=None, check: bool = True):
        c = self.cfgs[member]
        if out is None:
            out = [np.empty((c.ny, c.nx), dtype=np.float64) for _ in range(6)]
        p, ld, where, keep = _ptrs(out, c.nx, c.ny, out=True)
        rc = lib().chimera_batch_get_state(self._h, member, *p, ld, where)
        if check:
            _check(rc, "get_state")
        return out

    def get_stage_buffer(self, b: int):
        c = self.cfgs[0]
        out = [np.empty((c.ny, c.nx), dtype=np.float64) for _ in range(6)]
        p, ld, where, keep = _ptrs(out, c.nx, c.ny, out=True)
        _check(lib().chimera_get_stage_buffer(self._h, b, *p, ld, where), "get_stage_buffer")
        return out

    def set_time(self, t: float, output_count: int = 1, member: int = 0):
        _check(lib().chimera_batch_set_time(self._h, member, float(t), int(output_count)), "set_time")

    def step(self, nsteps: int = 1):
        _check(lib().chimera_step(self._h, int(nsteps)), "step")

    def step_host(self, inputs: Sequence, out=None):
        """One step on host arrays (chimera_step_host): ``inputs`` (six numpy
        arrays or CPU tensors, pinned for copy overlap) in, the new state to
        ``out`` (default: new numpy arrays; may be ``inputs``)."""
        c = self.cfgs[0]
        if out is None:
            out = [np.empty((c.ny, c.nx), dtype=np.float64) for _ in range(6)]
        pi, ld_i, wi, keep_i = _ptrs(inputs, c.nx, c.ny)
        po, ld_o, wo, keep_o = _ptrs(out, c.nx, c.ny, out=True)
        if wi != HOST or wo != HOST or ld_i != ld_o:
            raise ValueError("step_host takes host arrays with one pitch")
        P6 = C.c_void_p * 6
        _check(lib().chimera_step_host(self._h, P6(*[p.value for p in pi]), P6(*[p.value for p in po]), ld_i),
               "step_host")
        return out

    def advance(self, max_steps: int = 10 ** 9) -> int:
        n = C.c_int(0)
        _check(lib().chimera_advance(self._h, int(max_steps), C.byref(n)), "advance")
        return n.value

    def advance_output(self, max_steps: int = 10 ** 9) -> int:
        """Run to the next output time (or t_end): stops after the step that
        reaches it, where the reference writes a snapshot."""
        n = C.c_int(0)
        _check(lib().chimera_advance_output(self._h, int(max_steps), C.byref(n)), "advance_output")
        return n.value

    def stage(self, k: int, dt: float):
        _check(lib().chimera_stage(self._h, int(k), float(dt)), "stage")

    def diag(self, member: int = 0) -> dict:
        d = CDiag()
        _check(lib().chimera_batch_diag(self._h, member, C.byref(d)), "diag")
        return {f: getattr(d, f) for f, _ in CDiag._fields_}

    def set_counters(self, on: bool = True):
        _check(lib().chimera_set_counters(self._h, int(bool(on))), "set_counters")

    def set_graph_steps(self, n: int):
        _check(lib().chimera_set_graph_steps(self._h, int(n)), "set_graph_steps")

    def set_profiling(self, on: bool = True):
        _check(lib().chimera_set_profiling(self._h, int(bool(on))), "set_profiling")

    def get_profile(self, reset: bool = True) -> dict:
        """Device ms and launch counts of the CFL and the three stage kernels."""
        ms = (C.c_double * 4)()
        n = (C.c_longlong * 4)()
        _check(lib().chimera_get_profile(self._h, ms, n, int(bool(reset))), "get_profile")
        names = ("cfl", "stage1", "stage2", "stage3")
        return {k: {"ms": ms[i], "launches": n[i]} for i, k in enumerate(names)}

    def autotune(self, reps: int = 3):
        """Time every tile variant on the current state; keep the fastest."""
        v = C.c_int()
        ms = C.c_double()
        _check(lib().chimera_autotune(self._h, int(reps), C.byref(v), C.byref(ms)), "autotune")
        return v.value, ms.value

    def variant_count(self) -> int:
        return lib().chimera_variant_count(self._h)

    def set_variant(self, v: int):
        _check(lib().chimera_set_variant(self._h, int(v)), "set_variant")

    # ---- y-slab decomposition (chimera_halo_pack / _unpack, chimera_refresh_dt,
    # chimera_set_dt_device): asynchronous on the handle's stream, device tensors only
    @staticmethod
    def _dev_ptr(t):
        if t is None:
            return None
        if not (hasattr(t, "is_cuda") and t.is_cuda and t.is_contiguous()):
            raise ValueError("expected a contiguous CUDA tensor")
        return C.c_void_p(t.data_ptr())

    def halo_pack(self, rows: int, lo=None, hi=None):
        _check(lib().chimera_halo_pack(self._h, int(rows), self._dev_ptr(lo), self._dev_ptr(hi)), "halo_pack")

    def halo_unpack(self, rows: int, lo=None, hi=None):
        _check(lib().chimera_halo_unpack(self._h, int(rows), self._dev_ptr(lo), self._dev_ptr(hi)), "halo_unpack")

    def slab_ghost_rows(self, ghost_lo: int, ghost_hi: int):
        _check(lib().chimera_slab_ghost_rows(self._h, int(ghost_lo), int(ghost_hi)), "slab_ghost_rows")

    def refresh_dt(self, dt=None):
        _check(lib().chimera_refresh_dt(self._h, self._dev_ptr(dt)), "refresh_dt")

    def get_dt_device(self, dt):
        _check(lib().chimera_get_dt_device(self._h, self._dev_ptr(dt)), "get_dt_device")

    def set_dt_device(self, dt):
        _check(lib().chimera_set_dt_device(self._h, self._dev_ptr(dt)), "set_dt_device")

    def variant(self):
        v, tx, ty, nt = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        _check(lib().chimera_get_variant(self._h, C.byref(v), C.byref(tx), C.byref(ty), C.byref(nt)),
               "get_variant")
        return {"variant": v.value, "tile": (tx.value, ty.value), "threads": nt.value}
