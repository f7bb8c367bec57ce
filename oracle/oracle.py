"""ctypes binding of the CPU oracle (``oracle/chimera_oracle.c``).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA path.  Only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline / reference legs of
``bench.py`` import this module; the product package never does.

Each wrapper follows one reference routine (cited on the C side) and takes /
returns numpy float64 arrays shaped ``(ny, nx)`` (row-major, x fastest), which
is the memory layout of the Fortran ``real(8) (nx, ny)`` arrays.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

BC_PERIODIC, BC_FIXED, BC_OUTFLOW, BC_INFLOW = 1, 2, 3, 4
RUSANOV, HLLE, HLLD = 1, 2, 3
VAN_LEER, MC = 1, 2


class OrcCfg(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int),
        ("dx", C.c_double), ("dy", C.c_double),
        ("gamma", C.c_double), ("courant", C.c_double),
        ("t_out", C.c_double), ("t_end", C.c_double),
        ("bc_xlo", C.c_int), ("bc_xhi", C.c_int), ("bc_ylo", C.c_int), ("bc_yhi", C.c_int),
        ("riemann", C.c_int), ("limiter", C.c_int),
        ("slope_limiting", C.c_int), ("mood", C.c_int),
    ]


@dataclass
class Config:
    """Solver configuration; defaults are the reference's build-time switches
    (src/mhd_config.f90:16-62)."""
    nx: int
    ny: int
    dx: float
    dy: float
    gamma: float
    courant: float = 0.3
    t_out: float = 0.01
    t_end: float = 1.0
    bc: tuple = (BC_PERIODIC,) * 4  # xlo, xhi, ylo, yhi
    riemann: int = RUSANOV
    limiter: int = MC
    slope_limiting: bool = True
    mood: bool = True


def _c(cfg) -> OrcCfg:
    """Any object with the solver-config attributes (oracle.Config or the
    package's SolverConfig) -> the C struct."""
    return OrcCfg(int(cfg.nx), int(cfg.ny), float(cfg.dx), float(cfg.dy), float(cfg.gamma),
                  float(cfg.courant), float(cfg.t_out), float(cfg.t_end),
                  int(cfg.bc[0]), int(cfg.bc[1]), int(cfg.bc[2]), int(cfg.bc[3]),
                  int(cfg.riemann), int(cfg.limiter), int(bool(cfg.slope_limiting)),
                  int(bool(cfg.mood)))


_lib = None


def build() -> str:
    """Compile the oracle with its Makefile (gcc, -ffp-contract=off)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = C.CDLL(LIB_PATH)
        _lib.orc_cfl_dt.restype = C.c_double
        _lib.orc_run.restype = C.c_int
        _lib.orc_max_threads.restype = C.c_int
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _new(cfg: Config, pad: int = 0) -> np.ndarray:
    return np.zeros((cfg.ny + pad, cfg.nx + pad), dtype=np.float64)


def set_omp_mode(mode: int) -> None:
    """0 serial, 1 the reference's three OpenMP loops, 2 every loop."""
    lib().orc_set_omp_mode(int(mode))


def max_threads() -> int:
    return int(lib().orc_max_threads())


def set_threads(n: int) -> None:
    """Thread count of the OpenMP loops, overriding OMP_NUM_THREADS."""
    lib().orc_set_threads(int(n))


# --- routine-level wrappers (names follow the reference) ----------------------

def average_face_to_cell_B(cfg, b_x, b_y):
    Bx, By = _new(cfg), _new(cfg)
    lib().orc_average_face_to_cell_B(C.byref(_c(cfg)), _p(b_x), _p(b_y), _p(Bx), _p(By))
    return Bx, By


def compute_curl_2d(cfg, Az):
    bx, by = _new(cfg), _new(cfg)
    lib().orc_compute_curl_2d(C.byref(_c(cfg)), _p(Az), _p(bx), _p(by))
    return bx, by


def compute_divB(cfg, bx, by):
    d = _new(cfg)
    lib().orc_compute_divB(C.byref(_c(cfg)), _p(bx), _p(by), _p(d))
    return d


def get_conserved(cfg, rho, vx, vy, P, Bx, By):
    out = [_new(cfg) for _ in range(4)]
    vol = C.c_double(cfg.dx * cfg.dy)
    lib().orc_get_conserved(C.byref(_c(cfg)), _p(rho), _p(vx), _p(vy), _p(P), _p(Bx), _p(By),
                            vol, *[_p(o) for o in out])
    return tuple(out)


def get_primitive(cfg, Mass, Momx, Momy, Energy, Bx, By):
    out = [_new(cfg) for _ in range(4)]
    vol = C.c_double(cfg.dx * cfg.dy)
    lib().orc_get_primitive(C.byref(_c(cfg)), _p(Mass), _p(Momx), _p(Momy), _p(Energy),
                            _p(Bx), _p(By), vol, *[_p(o) for o in out])
    return tuple(out)


def apply_conserved_floors(cfg, Mass, Momx, Momy, Energy, Bx, By):
    M, Mx, My, E = (np.array(a, dtype=np.float64, copy=True) for a in (Mass, Momx, Momy, Energy))
    vol = C.c_double(cfg.dx * cfg.dy)
    lib().orc_apply_conserved_floors(C.byref(_c(cfg)), _p(M), _p(Mx), _p(My), _p(E),
                                     _p(Bx), _p(By), vol)
    return M, Mx, My, E


def fill_ghost_cells(cfg, f):
    pad = _new(cfg, 2)
    lib().orc_fill_ghost_cells(C.byref(_c(cfg)), _p(np.ascontiguousarray(f)), _p(pad))
    return pad


def compute_gradients(cfg, f_pad):
    fdx, fdy = _new(cfg), _new(cfg)
    lib().orc_compute_gradients(C.byref(_c(cfg)), _p(f_pad), _p(fdx), _p(fdy))
    return fdx, fdy


def apply_slope_limiter(cfg, f_pad):
    fdx, fdy = _new(cfg), _new(cfg)
    lib().orc_apply_slope_limiter(C.byref(_c(cfg)), _p(f_pad), _p(fdx), _p(fdy))
    return fdx, fdy


def reconstruction(cfg, f, f_dx, f_dy, rho_or_p: bool):
    out = [_new(cfg) for _ in range(4)]
    lib().orc_reconstruction(C.byref(_c(cfg)), _p(f), _p(f_dx), _p(f_dy),
                             *[_p(o) for o in out], C.c_int(int(rho_or_p)))
    return tuple(out)


def compute_fluxes(cfg, rho_L, rho_R, vx_L, vx_R, vy_L, vy_R, P_L, P_R, Bx_L, Bx_R, By_L, By_R):
    out = [_new(cfg) for _ in range(5)]
    args = [rho_L, rho_R, vx_L, vx_R, vy_L, vy_R, P_L, P_R, Bx_L, Bx_R, By_L, By_R]
    args = [np.ascontiguousarray(a, dtype=np.float64) for a in args]
    lib().orc_compute_fluxes(C.byref(_c(cfg)), *[_p(a) for a in args], *[_p(o) for o in out])
    return tuple(out)


def update_conserved(cfg, F, fX, fY, dt):
    F = np.array(F, dtype=np.float64, copy=True)
    lib().orc_update_conserved(C.byref(_c(cfg)), _p(F), _p(fX), _p(fY), C.c_double(dt))
    return F


def constrained_transport(cfg, bx, by, fByX, fBxY, dt):
    bx = np.array(bx, dtype=np.float64, copy=True)
    by = np.array(by, dtype=np.float64, copy=True)
    lib().orc_constrained_transport(C.byref(_c(cfg)), _p(bx), _p(by), _p(fByX), _p(fBxY),
                                    C.c_double(dt))
    return bx, by


def cfl_dt(cfg, rho, vx, vy, P, Bx, By, t=0.0, output_count=1):
    return float(lib().orc_cfl_dt(C.byref(_c(cfg)), _p(rho), _p(vx), _p(vy), _p(P), _p(Bx), _p(By),
                                  C.c_double(t), C.c_int(output_count)))


# --- composite entry points ---------------------------------------------------

class State:
    """Conserved state (Mass, Momx, Momy, Energy, b_x, b_y) plus the time-loop
    counters of src/main.f90:61-63."""

    FIELDS = ("Mass", "Momx", "Momy", "Energy", "b_x", "b_y")

    def __init__(self, arrays, t=0.0, output_count=1):
        self.a = [np.array(x, dtype=np.float64, copy=True, order="C") for x in arrays]
        self.t = float(t)
        self.output_count = int(output_count)

    def copy(self):
        return State(self.a, self.t, self.output_count)


def run(cfg, state: State, nsteps: int, dt_fixed=None):
    """Advance ``state`` in place by up to ``nsteps`` RK3 steps (stops once
    t >= t_end).  Returns the list of dt values used."""
    t = C.c_double(state.t)
    oc = C.c_int(state.output_count)
    dt_log = np.zeros(max(nsteps, 1), dtype=np.float64)
    fixed = None
    if dt_fixed is not None:
        fixed = np.ascontiguousarray(dt_fixed, dtype=np.float64)
    taken = lib().orc_run(C.byref(_c(cfg)), *[_p(x) for x in state.a], C.byref(t), C.byref(oc),
                          C.c_int(nsteps), _p(fixed) if fixed is not None else None, _p(dt_log))
    state.t, state.output_count = t.value, oc.value
    return dt_log[:taken].copy()


def stage(cfg, k, dt, state_arrays, u0_arrays):
    out = [np.array(x, dtype=np.float64, copy=True) for x in state_arrays]
    u0 = [np.ascontiguousarray(x, dtype=np.float64) for x in u0_arrays]
    lib().orc_stage(C.byref(_c(cfg)), C.c_int(k), C.c_double(dt), *[_p(x) for x in out],
                    *[_p(x) for x in u0])
    return out


def stage_fluxes(cfg, state_arrays):
    fx = [_new(cfg) for _ in range(5)]
    fy = [_new(cfg) for _ in range(5)]
    s = [np.ascontiguousarray(x, dtype=np.float64) for x in state_arrays]
    lib().orc_stage_fluxes(C.byref(_c(cfg)), *[_p(x) for x in s], *[_p(x) for x in fx],
                           *[_p(x) for x in fy])
    return fx, fy


def primitives(cfg, state_arrays):
    out = [_new(cfg) for _ in range(6)]
    s = [np.ascontiguousarray(x, dtype=np.float64) for x in state_arrays]
    lib().orc_primitives(C.byref(_c(cfg)), *[_p(x) for x in s], *[_p(o) for o in out])
    return tuple(out)  # rho, vx, vy, P_total, Bx, By
