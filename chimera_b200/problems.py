"""Initial states for the benchmark problems (host-side, numpy FP64).

Initial conditions are inputs to the per-step path, not part of it.  The
reference's own set-ups are followed where a workload uses them
(Orszag-Tang ``src/mhd_init.f90:296-311``, rotor ``:399-450``, field loop
``:360-391``); the other workloads (GRF ensemble, field loop on [0,2]x[0,1],
Kelvin-Helmholtz on [0,1]x[-1,1]) are seeded synthetic states with the shapes
and value ranges of their specification.

Every generator returns ``(cfg, arrays)`` where ``cfg`` is a
:class:`chimera_b200.config.SolverConfig` and ``arrays`` is the conserved state
``[Mass, Momx, Momy, Energy, b_x, b_y]`` as ``(ny, nx)`` float64 arrays
(x fastest, i.e. the Fortran ``(nx, ny)`` column-major layout).
"""
from __future__ import annotations

import math

import numpy as np

from .config import (BC_OUTFLOW, BC_PERIODIC, HLLE, MC, RUSANOV, VAN_LEER, HLLD,
                     SolverConfig)

# src/mhd_config.f90:54-56 (the reference's literal constants)
PI = 3.1415926535897932
TWO_PI = 6.2831853071795865
FOUR_PI = 12.566370614359173
RHO_FLOOR = 1.0e-12
P_FLOOR = 1.0e-12


def curl_2d(Az, dx, dy, periodic_x=True, periodic_y=True):
    """Face B from a cell-centred A_z, following compute_curl_2d
    (src/mhd_field_ops.f90:15-57): backward differences, BC-aware first row."""
    inv_dx = 1.0 / dx
    inv_dy = 1.0 / dy
    bx = np.empty_like(Az)
    by = np.empty_like(Az)
    bx[1:, :] = (Az[1:, :] - Az[:-1, :]) * inv_dy
    bx[0, :] = (Az[0, :] - Az[-1, :]) * inv_dy if periodic_y else bx[1, :]
    by[:, 1:] = -((Az[:, 1:] - Az[:, :-1]) * inv_dx)
    by[:, 0] = -((Az[:, 0] - Az[:, -1]) * inv_dx) if periodic_x else by[:, 1]
    return bx, by


def face_to_cell(b_x, b_y, periodic_x=True, periodic_y=True):
    """Cell-centred B from face B (average_face_to_cell_B,
    src/mhd_field_ops.f90:120-156)."""
    Bx = np.empty_like(b_x)
    By = np.empty_like(b_y)
    Bx[:, 1:] = 0.5 * (b_x[:, 1:] + b_x[:, :-1])
    Bx[:, 0] = 0.5 * (b_x[:, 0] + b_x[:, -1]) if periodic_x else b_x[:, 0]
    By[1:, :] = 0.5 * (b_y[1:, :] + b_y[:-1, :])
    By[0, :] = 0.5 * (b_y[0, :] + b_y[-1, :]) if periodic_y else b_y[0, :]
    return Bx, By


def get_conserved(rho, vx, vy, P, Bx, By, gamma, vol):
    """Primitive -> conserved (get_conserved, src/mhd_change_states.f90:16-58).
    P is the TOTAL pressure p + B^2/2."""
    rho_cp = np.maximum(rho, RHO_FLOOR)
    P_cp = np.maximum(P, P_FLOOR)
    Mass = rho_cp * vol
    Momx = Mass * vx
    Momy = Mass * vy
    halfB2 = 0.5 * (Bx * Bx + By * By)
    Energy = (((P_cp - halfB2) / (gamma - 1.0) + (0.5 * rho_cp) * (vx * vx + vy * vy)) + halfB2) * vol
    return Mass, Momx, Momy, Energy


def _cell_centres(n, lo, d):
    return (np.arange(1, n + 1, dtype=np.float64) - 0.5) * d + lo


def _finish(cfg, rho, vx, vy, p_thermal, b_x, b_y):
    px = cfg.bc[0] == BC_PERIODIC
    py = cfg.bc[2] == BC_PERIODIC
    Bx, By = face_to_cell(b_x, b_y, px, py)
    P = p_thermal + 0.5 * (Bx * Bx + By * By)
    M, Mx, My, E = get_conserved(rho, vx, vy, P, Bx, By, cfg.gamma, cfg.dx * cfg.dy)
    return [np.ascontiguousarray(a, dtype=np.float64) for a in (M, Mx, My, E, b_x, b_y)]


def orszag_tang(n=256, riemann=RUSANOV, limiter=MC, mood=True, t_end=0.5):
    """Orszag-Tang vortex on the unit square, periodic (setup_OT_vortex,
    src/mhd_init.f90:296-311)."""
    dx = 1.0 / n
    cfg = SolverConfig(nx=n, ny=n, dx=dx, dy=dx, gamma=5.0 / 3.0, riemann=riemann,
                       limiter=limiter, mood=mood, t_end=t_end, bc=(BC_PERIODIC,) * 4)
    xlin = _cell_centres(n, 0.0, dx)
    X = np.broadcast_to(xlin[None, :], (n, n))
    Y = np.broadcast_to(xlin[:, None], (n, n))
    rho = np.full((n, n), 25.0 / (36.0 * PI))
    p = np.full((n, n), 5.0 / (12.0 * PI))
    vx = -np.sin(TWO_PI * Y)
    vy = np.sin(TWO_PI * X)
    Az = np.cos(FOUR_PI * X) / (FOUR_PI * math.sqrt(FOUR_PI)) + \
        np.cos(TWO_PI * Y) / (TWO_PI * math.sqrt(FOUR_PI))
    b_x, b_y = curl_2d(Az, dx, dx)
    return cfg, _finish(cfg, rho, vx, vy, p, b_x, b_y)


def rotor(n=1024, riemann=HLLE, limiter=MC, mood=True, t_end=0.15):
    """MHD rotor on the unit square with outflow on every side
    (setup_rotor, src/mhd_init.f90:399-450), gamma = 1.4."""
    dx = 1.0 / n
    cfg = SolverConfig(nx=n, ny=n, dx=dx, dy=dx, gamma=1.4, riemann=riemann, limiter=limiter,
                       mood=mood, t_end=t_end, bc=(BC_OUTFLOW,) * 4)
    xlin = _cell_centres(n, 0.0, dx)
    X = np.broadcast_to(xlin[None, :], (n, n))
    Y = np.broadcast_to(xlin[:, None], (n, n))
    x0 = y0 = 0.5
    r0, r1, u0 = 0.1, 0.115, 2.0
    rx = X - x0
    ry = Y - y0
    r = np.sqrt(rx * rx + ry * ry)
    rho = np.ones((n, n))
    vx = np.zeros((n, n))
    vy = np.zeros((n, n))
    core = r <= r0
    rho[core] = 10.0
    vx[core] = -u0 * (ry[core] / r0)
    vy[core] = u0 * (rx[core] / r0)
    taper = (~core) & (r < r1)
    f = (r1 - r[taper]) / (r1 - r0)
    rho[taper] = 1.0 + 9.0 * f
    rt = r[taper]
    vx[taper] = np.where(rt > 0, -f * u0 * (ry[taper] / np.where(rt > 0, rt, 1.0)), 0.0)
    vy[taper] = np.where(rt > 0, f * u0 * (rx[taper] / np.where(rt > 0, rt, 1.0)), 0.0)
    p = np.ones((n, n))
    b_x = np.full((n, n), 5.0 / math.sqrt(4.0 * PI))
    b_y = np.zeros((n, n))
    return cfg, _finish(cfg, rho, vx, vy, p, b_x, b_y)


def field_loop(nx=512, ny=512, lx=2.0, ly=1.0, v=(2.0, 1.0), riemann=HLLE, limiter=VAN_LEER,
               mood=True, t_end=1.0):
    """Field-loop advection: rho = p = 1, uniform v, A_z = 1e-3 (0.3 - r) for
    r < 0.3 about the box centre, gamma = 5/3, periodic.  The reference set-up
    (src/mhd_init.f90:360-391) is the unit-square case with v = (-2, -1)."""
    dx = lx / nx
    dy = ly / ny
    cfg = SolverConfig(nx=nx, ny=ny, dx=dx, dy=dy, gamma=5.0 / 3.0, riemann=riemann,
                       limiter=limiter, mood=mood, t_end=t_end, bc=(BC_PERIODIC,) * 4)
    X = np.broadcast_to(_cell_centres(nx, 0.0, dx)[None, :], (ny, nx))
    Y = np.broadcast_to(_cell_centres(ny, 0.0, dy)[:, None], (ny, nx))
    r = np.sqrt((X - 0.5 * lx) ** 2 + (Y - 0.5 * ly) ** 2)
    Az = np.where(r < 0.3, 1.0e-3 * (0.3 - r), 0.0)
    b_x, b_y = curl_2d(Az, dx, dy)
    rho = np.ones((ny, nx))
    vx = np.full((ny, nx), float(v[0]))
    vy = np.full((ny, nx), float(v[1]))
    return cfg, _finish(cfg, rho, vx, vy, np.ones((ny, nx)), b_x, b_y)


def kelvin_helmholtz(n=4096, riemann=HLLD, limiter=MC, mood=True, seed=0, t_end=1e30):
    """Magnetised Kelvin-Helmholtz on [0,1] x [-1,1], periodic, gamma = 1.4:
    rho = 1, p = 2.5, vx = 0.5 tanh(y/0.05) mirrored at |y| = 1/2 so the
    profile is periodic, vy = 0.01 sin(2 pi x) exp(-y^2/0.01) plus seeded
    uniform noise of amplitude 1e-3, Bx = 0.1."""
    nx = ny = n
    dx = 1.0 / nx
    dy = 2.0 / ny
    cfg = SolverConfig(nx=nx, ny=ny, dx=dx, dy=dy, gamma=1.4, riemann=riemann, limiter=limiter,
                       mood=mood, t_end=t_end, bc=(BC_PERIODIC,) * 4)
    x = _cell_centres(nx, 0.0, dx)
    y = _cell_centres(ny, -1.0, dy)
    X = np.broadcast_to(x[None, :], (ny, nx))
    Y = np.broadcast_to(y[:, None], (ny, nx))
    a = 0.05
    ym = np.where(Y > 0.5, 1.0 - Y, np.where(Y < -0.5, -1.0 - Y, Y))
    vx = 0.5 * np.tanh(ym / a)
    rng = np.random.Generator(np.random.Philox(seed))
    vy = 0.01 * np.sin(2.0 * np.pi * X) * np.exp(-Y * Y / 0.01) + \
        1.0e-3 * rng.uniform(-1.0, 1.0, size=(ny, nx))
    b_x = np.full((ny, nx), 0.1)
    b_y = np.zeros((ny, nx))
    return cfg, _finish(cfg, np.ones((ny, nx)), vx, vy, np.full((ny, nx), 2.5), b_x, b_y)


def _rbf_smooth(noise, length, d):
    """Periodic convolution of white noise with exp(-r^2 / (2 l^2)) (FFT)."""
    ny, nx = noise.shape
    kx = 2.0 * np.pi * np.fft.fftfreq(nx, d=d)
    ky = 2.0 * np.pi * np.fft.fftfreq(ny, d=d)
    k2 = ky[:, None] ** 2 + kx[None, :] ** 2
    return np.real(np.fft.ifft2(np.fft.fft2(noise) * np.exp(-0.5 * length * length * k2)))


def grf_member(n, seed, length=0.1, cf_cap=3.0, mach=None, beta=None):
    """One GRF ensemble member on the periodic unit square: stream function psi
    and vector potential A_z are white Gaussian noise smoothed by a Gaussian
    RBF of length ``length``; v = curl psi scaled to rms V0 ~ U[0.5, 2];
    B = curl A_z (face centred) scaled to rms B0 ~ U[0.2, 1]; rho = p = 1;
    gamma ~ U[1.4, 5/3]; where max(c_f + |v|) exceeds cf_cap the velocities are
    scaled by cf_cap / max(c_f + |v|) and B is left alone (the cap step of
    src/mhd_init.f90:811-829, which can leave the maximum above cf_cap when
    c_f is large).  Philox-seeded.

    ``mach`` / ``beta`` override the drawn rms speed / field with a target
    sonic Mach number and plasma beta, V0 = mach sqrt(gamma) and
    B0 = sqrt(2 / beta) at rho = p = 1 (the counterpart of the reference's
    M_s and beta overrides, exercised by tests/stress/test_stress.py:113-234);
    the draws are still made, so the rest of the member is the seed's."""
    rng = np.random.Generator(np.random.Philox(seed))
    gamma = rng.uniform(1.4, 5.0 / 3.0)
    V0 = rng.uniform(0.5, 2.0)
    B0 = rng.uniform(0.2, 1.0)
    if mach is not None:
        V0 = float(mach) * math.sqrt(gamma)
    if beta is not None:
        B0 = math.sqrt(2.0 / float(beta))
    dx = 1.0 / n
    psi = _rbf_smooth(rng.standard_normal((n, n)), length, dx)
    Az = _rbf_smooth(rng.standard_normal((n, n)), length, dx)
    vx = (np.roll(psi, -1, axis=0) - np.roll(psi, 1, axis=0)) / (2.0 * dx)
    vy = -(np.roll(psi, -1, axis=1) - np.roll(psi, 1, axis=1)) / (2.0 * dx)
    vrms = math.sqrt(float(np.mean(vx * vx + vy * vy)))
    vx *= V0 / vrms
    vy *= V0 / vrms
    b_x, b_y = curl_2d(Az, dx, dx)
    Bx, By = face_to_cell(b_x, b_y)
    brms = math.sqrt(float(np.mean(Bx * Bx + By * By)))
    b_x *= B0 / brms
    b_y *= B0 / brms
    Bx, By = face_to_cell(b_x, b_y)
    rho = np.ones((n, n))
    p = np.ones((n, n))
    cf = np.sqrt(gamma * p / rho + (Bx * Bx + By * By) / rho)
    top = float(np.max(cf + np.sqrt(vx * vx + vy * vy)))
    if top > cf_cap:
        vx *= cf_cap / top
        vy *= cf_cap / top
    cfg = SolverConfig(nx=n, ny=n, dx=dx, dy=dx, gamma=gamma, riemann=RUSANOV, limiter=MC,
                       mood=True, t_end=1e30, bc=(BC_PERIODIC,) * 4)
    return cfg, _finish(cfg, rho, vx, vy, p, b_x, b_y)


def grf_ensemble_sizes(scale=1):
    """Member sizes of the GRF ensemble: 256 at 128^2, 192 at 256^2, 64 at
    512^2 (33.55 M cells).  ``scale`` divides the member counts for smaller
    test ensembles."""
    sizes = [128] * (256 // scale) + [256] * (192 // scale) + [512] * (64 // scale)
    return sizes
