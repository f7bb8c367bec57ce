"""The reference's module routines on the GPU, one kernel each
(``chimera_op_*`` in include/chimera_gpu.h), with the Fortran names and
argument meaning.  Arrays are CUDA float64 tensors shaped (ny, nx); outputs
are returned as new tensors (the Fortran intent(out) arguments), in-place
routines update their intent(inout) arguments.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import gpu
from .config import SolverConfig

_bound = False


def _lib():
    global _bound
    L = gpu.lib()
    if not _bound:
        P = C.c_void_p
        cp = C.POINTER(gpu.CCfg)
        sig = {
            "chimera_op_average_face_to_cell_B": [cp, P, P, P, P, P],
            "chimera_op_get_primitive": [cp] + [P] * 10 + [P],
            "chimera_op_get_conserved": [cp] + [P] * 10 + [P],
            "chimera_op_apply_conserved_floors": [cp] + [P] * 6 + [P],
            "chimera_op_fill_ghost_cells": [cp, P, P, P],
            "chimera_op_compute_gradients": [cp, P, P, P, P],
            "chimera_op_apply_slope_limiter": [cp, P, P, P, P],
            "chimera_op_reconstruction": [cp] + [P] * 7 + [C.c_int, P],
            "chimera_op_thermal_pressure_check": [cp, P * 24, P * 6, P],
            "chimera_op_compute_fluxes": [cp, P * 12, P * 5, P],
            "chimera_op_update_conserved": [cp, P, P, P, C.c_double, P],
            "chimera_op_constrained_transport": [cp, P, P, P, P, C.c_double, P, P],
            "chimera_op_compute_curl_2d": [cp, P, P, P, P],
            "chimera_op_compute_divB": [cp, P, P, P, P],
        }
        for name, args in sig.items():
            getattr(L, name).argtypes = args
        _bound = True
    return L


def _p(t):
    if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
        raise ValueError("expected contiguous CUDA float64 tensors")
    return C.c_void_p(t.data_ptr())


def _call(name, cfg, *args):
    ccfg = gpu.to_ccfg(cfg)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = getattr(_lib(), name)(C.byref(ccfg), *args, stream)
    if rc != 0:
        raise gpu.ChimeraError(rc, name)


def _like(t, n=1):
    return [torch.empty_like(t) for _ in range(n)]


def average_face_to_cell_B(cfg: SolverConfig, b_x, b_y):
    Bx, By = _like(b_x, 2)
    _call("chimera_op_average_face_to_cell_B", cfg, _p(b_x), _p(b_y), _p(Bx), _p(By))
    return Bx, By


def get_primitive(cfg, Mass, Momx, Momy, Energy, Bx, By):
    out = _like(Mass, 4)
    _call("chimera_op_get_primitive", cfg, *[_p(t) for t in (Mass, Momx, Momy, Energy, Bx, By, *out)])
    return tuple(out)


def get_conserved(cfg, rho, vx, vy, P, Bx, By):
    out = _like(rho, 4)
    _call("chimera_op_get_conserved", cfg, *[_p(t) for t in (rho, vx, vy, P, Bx, By, *out)])
    return tuple(out)


def apply_conserved_floors(cfg, Mass, Momx, Momy, Energy, Bx, By):
    """In place on Mass..Energy (intent(inout)); also returned."""
    _call("chimera_op_apply_conserved_floors", cfg, *[_p(t) for t in (Mass, Momx, Momy, Energy, Bx, By)])
    return Mass, Momx, Momy, Energy


def fill_ghost_cells(cfg, f):
    pad = torch.empty((f.shape[0] + 2, f.shape[1] + 2), dtype=f.dtype, device=f.device)
    _call("chimera_op_fill_ghost_cells", cfg, _p(f), _p(pad))
    return pad


def compute_gradients(cfg, f_pad):
    ny, nx = f_pad.shape[0] - 2, f_pad.shape[1] - 2
    fdx = torch.empty((ny, nx), dtype=f_pad.dtype, device=f_pad.device)
    fdy = torch.empty_like(fdx)
    _call("chimera_op_compute_gradients", cfg, _p(f_pad), _p(fdx), _p(fdy))
    return fdx, fdy


def apply_slope_limiter(cfg, f_pad):
    ny, nx = f_pad.shape[0] - 2, f_pad.shape[1] - 2
    fdx = torch.empty((ny, nx), dtype=f_pad.dtype, device=f_pad.device)
    fdy = torch.empty_like(fdx)
    _call("chimera_op_apply_slope_limiter", cfg, _p(f_pad), _p(fdx), _p(fdy))
    return fdx, fdy


def reconstruction(cfg, f, f_dx, f_dy, rho_or_p: bool):
    out = _like(f, 4)
    _call("chimera_op_reconstruction", cfg, _p(f), _p(f_dx), _p(f_dy), *[_p(t) for t in out],
          C.c_int(int(rho_or_p)))
    return tuple(out)


def thermal_pressure_check(cfg, P_f, Bx_f, By_f, rho_f, vx_f, vy_f, rho0, vx0, vy0, P0, Bx0, By0):
    """In place on the face arrays; *_f are 4-tuples (XL, XR, YL, YR)."""
    faces = []
    for s in range(4):
        faces += [P_f[s], Bx_f[s], By_f[s], rho_f[s], vx_f[s], vy_f[s]]
    cell = [P0, Bx0, By0, rho0, vx0, vy0]
    _call("chimera_op_thermal_pressure_check", cfg, (C.c_void_p * 24)(*[t.data_ptr() for t in faces]),
          (C.c_void_p * 6)(*[t.data_ptr() for t in cell]))


def compute_fluxes(cfg, rho_L, rho_R, vx_L, vx_R, vy_L, vy_R, P_L, P_R, Bx_L, Bx_R, By_L, By_R):
    ins = [rho_L, rho_R, vx_L, vx_R, vy_L, vy_R, P_L, P_R, Bx_L, Bx_R, By_L, By_R]
    for t in ins:
        _p(t)
    out = _like(rho_L, 5)
    _call("chimera_op_compute_fluxes", cfg, (C.c_void_p * 12)(*[t.data_ptr() for t in ins]),
          (C.c_void_p * 5)(*[t.data_ptr() for t in out]))
    return tuple(out)


def update_conserved(cfg, F, flux_X, flux_Y, dt):
    """In place on F (intent(inout)); also returned."""
    _call("chimera_op_update_conserved", cfg, _p(F), _p(flux_X), _p(flux_Y), C.c_double(dt))
    return F


def constrained_transport(cfg, b_x, b_y, flux_By_X, flux_Bx_Y, dt):
    """In place on b_x, b_y (intent(inout)); also returned."""
    scratch = torch.empty_like(b_x)
    _call("chimera_op_constrained_transport", cfg, _p(b_x), _p(b_y), _p(flux_By_X), _p(flux_Bx_Y),
          C.c_double(dt), _p(scratch))
    return b_x, b_y


def compute_curl_2d(cfg, Az):
    bx, by = _like(Az, 2)
    _call("chimera_op_compute_curl_2d", cfg, _p(Az), _p(bx), _p(by))
    return bx, by


def compute_divB(cfg, b_x, b_y):
    d = torch.empty_like(b_x)
    _call("chimera_op_compute_divB", cfg, _p(b_x), _p(b_y), _p(d))
    return d
