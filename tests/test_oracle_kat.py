"""The reference's Fortran known-answer tests, ported onto the CPU oracle.

Each test cites the Fortran test it restates; tolerances are the reference's.
"""

import numpy as np
import pytest

from oracle.oracle import BC_OUTFLOW, BC_PERIODIC, Config

TWO_PI = 6.2831853071795865
FOUR_PI = 12.566370614359173


def _cfg(n, bc=(BC_PERIODIC,) * 4, gamma=5.0 / 3.0, dx=None):
    dx = dx if dx is not None else 1.0 / n
    return Config(nx=n, ny=n, dx=dx, dy=dx, gamma=gamma, bc=bc)


# --- tests/fortran/test_bcs.f90:15-97 ------------------------------------------
def _pattern(n=8):
    i = np.arange(1, n + 1, dtype=np.float64)
    return i[None, :] + 10.0 * i[:, None]          # f(i,j) = i + 10 j, (ny, nx)


def test_bcs_periodic(oracle):
    f = _pattern()
    pad = oracle.fill_ghost_cells(_cfg(8), f)
    tol = 1e-14
    assert np.max(np.abs(pad[1:-1, 0] - f[:, -1])) < tol      # left ghost = right col
    assert np.max(np.abs(pad[1:-1, -1] - f[:, 0])) < tol      # right ghost = left col
    assert np.max(np.abs(pad[0, 1:-1] - f[-1, :])) < tol      # bottom ghost = top row
    assert np.max(np.abs(pad[-1, 1:-1] - f[0, :])) < tol      # top ghost = bottom row
    assert np.max(np.abs(pad[1:-1, 1:-1] - f)) < tol          # interior unchanged
    assert abs(pad[0, 0] - f[-1, -1]) < tol                   # lower-left = f(N,N)


def test_bcs_outflow(oracle):
    f = _pattern()
    pad = oracle.fill_ghost_cells(_cfg(8, (BC_OUTFLOW,) * 4), f)
    tol = 1e-14
    assert np.max(np.abs(pad[1:-1, 0] - f[:, 0])) < tol
    assert np.max(np.abs(pad[1:-1, -1] - f[:, -1])) < tol
    assert np.max(np.abs(pad[0, 1:-1] - f[0, :])) < tol
    assert np.max(np.abs(pad[-1, 1:-1] - f[-1, :])) < tol
    assert abs(pad[0, 0] - f[0, 0]) < tol
    assert abs(pad[-1, -1] - f[-1, -1]) < tol


def test_bcs_mixed(oracle):
    f = _pattern()
    pad = oracle.fill_ghost_cells(_cfg(8, (BC_PERIODIC, BC_PERIODIC, BC_OUTFLOW, BC_OUTFLOW)), f)
    tol = 1e-14
    assert np.max(np.abs(pad[1:-1, 0] - f[:, -1])) < tol      # x periodic
    assert np.max(np.abs(pad[0, 1:-1] - f[0, :])) < tol       # y outflow
    assert abs(pad[0, 0] - f[0, -1]) < tol                    # x wraps, y doesn't


# --- tests/fortran/test_change_states.f90:14-104 -------------------------------
VOL = (1.0 / 64.0) ** 2


def _cs_cfg():
    # vol = (1/64)^2 as in the Fortran test
    return Config(nx=4, ny=4, dx=1.0 / 64.0, dy=1.0 / 64.0, gamma=5.0 / 3.0)


def test_change_states_round_trip(oracle):
    c = _cs_cfg()
    sh = (4, 4)
    rho, vx, vy = np.full(sh, 1.5), np.full(sh, 0.3), np.full(sh, -0.2)
    Bx, By = np.full(sh, 0.5), np.full(sh, 0.3)
    P = np.full(sh, 1.0 + 0.5 * (0.5 ** 2 + 0.3 ** 2))
    M, Mx, My, E = oracle.get_conserved(c, rho, vx, vy, P, Bx, By)
    r2, u2, v2, P2 = oracle.get_primitive(c, M, Mx, My, E, Bx, By)
    tol = 1e-10
    assert np.max(np.abs(r2 - rho)) < tol
    assert np.max(np.abs(u2 - vx)) < tol
    assert np.max(np.abs(v2 - vy)) < tol
    assert np.max(np.abs(P2 - P)) < tol


def test_change_states_density_floor(oracle):
    c = _cs_cfg()
    sh = (4, 4)
    rho, vx, vy, P = np.full(sh, 1e-20), np.ones(sh), np.zeros(sh), np.ones(sh)
    Bx, By = np.zeros(sh), np.zeros(sh)
    M, Mx, My, E = oracle.get_conserved(c, rho, vx, vy, P, Bx, By)
    r2, u2, _, _ = oracle.get_primitive(c, M, Mx, My, E, Bx, By)
    assert r2.min() >= 1e-12
    assert np.max(np.abs(u2)) < 1e6


def test_change_states_proportional_floor(oracle):
    c = _cs_cfg()
    sh = (4, 4)
    rho, vx, Bx = 1.0, 1.0e3, 0.5
    halfB2 = 0.5 * Bx * Bx
    KE = 0.5 * rho * vx * vx
    M = np.full(sh, rho * VOL)
    Mx = np.full(sh, rho * vx * VOL)
    My = np.zeros(sh)
    E = np.full(sh, (KE + halfB2) * VOL)
    _, _, _, P = oracle.get_primitive(c, M, Mx, My, E, np.full(sh, Bx), np.zeros(sh))
    floor = halfB2 + 1e-10 * (KE + halfB2)
    assert P.min() > 0.0
    assert P.min() >= floor * (1.0 - 1e-10)


# --- tests/fortran/test_field_ops.f90:16-127 -----------------------------------
def _grid32():
    n = 32
    dx = 1.0 / n
    x = (np.arange(1, n + 1) - 0.5) * dx
    return n, dx, x[None, :], x[:, None]


def test_div_curl_is_zero(oracle):
    n, dx, X, Y = _grid32()
    Az = np.sin(TWO_PI * X) * np.cos(TWO_PI * Y) + 0.3 * np.cos(FOUR_PI * X) * np.sin(TWO_PI * Y)
    c = _cfg(n)
    bx, by = oracle.compute_curl_2d(c, np.ascontiguousarray(Az))
    d = oracle.compute_divB(c, bx, by)
    assert np.max(np.abs(d[1:, 1:])) < 1e-13
    assert max(np.max(np.abs(d[:, 0])), np.max(np.abs(d[0, :]))) < 1e-13


@pytest.mark.parametrize("bc", [(BC_OUTFLOW,) * 4, (BC_PERIODIC, BC_PERIODIC, BC_OUTFLOW, BC_OUTFLOW)])
def test_div_curl_is_zero_nonperiodic(oracle, bc):
    """Same identity on the interior with outflow sides.  (The boundary copy of
    compute_curl_2d, src/mhd_field_ops.f90:214-228, does not make the first
    row/column divergence free, so only i,j >= 2 are checked.)"""
    n, dx, X, Y = _grid32()
    Az = np.sin(3.0 * X) * np.cos(2.0 * Y) + 0.3 * X * Y
    c = _cfg(n, bc)
    bx, by = oracle.compute_curl_2d(c, np.ascontiguousarray(Az))
    d = oracle.compute_divB(c, bx, by)
    assert np.max(np.abs(d[1:, 1:])) < 1e-12


def test_gradient_linear_exact(oracle):
    n, dx, X, Y = _grid32()
    f = np.ascontiguousarray(3.0 * X + 2.0 * Y)
    pad = oracle.fill_ghost_cells(_cfg(n), f)
    fdx, fdy = oracle.compute_gradients(_cfg(n), pad)
    assert np.max(np.abs(fdx[1:-1, 1:-1] - 3.0)) < 1e-13
    assert np.max(np.abs(fdy[1:-1, 1:-1] - 2.0)) < 1e-13


def test_gradient_sinusoid_second_order(oracle):
    n, dx, X, Y = _grid32()
    f = np.ascontiguousarray(np.sin(TWO_PI * X) * np.cos(TWO_PI * Y))
    pad = oracle.fill_ghost_cells(_cfg(n), f)
    fdx, fdy = oracle.compute_gradients(_cfg(n), pad)
    ex = TWO_PI * np.cos(TWO_PI * X) * np.cos(TWO_PI * Y)
    ey = -TWO_PI * np.sin(TWO_PI * X) * np.sin(TWO_PI * Y)
    assert np.max(np.abs(fdx - ex)) < 0.1
    assert np.max(np.abs(fdy - ey)) < 0.1
