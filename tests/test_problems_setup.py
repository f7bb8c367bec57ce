"""The host set-ups of chimera_b200.problems against the reference's set-up
routines: each initial state is rebuilt here from the reference's formulas and
constants (src/mhd_config.f90:54-56, cell centres (i - 1/2) dx of
src/main.f90:36-40), through the oracle's restatements of the reference
routines the set-ups call (compute_curl_2d, average_face_to_cell_B, and
get_conserved as src/main.f90:49 applies it), and must equal the package's
state bit for bit.  The rotor is rebuilt by the reference's per-cell loop.
The Kelvin-Helmholtz and adjoint field-loop workloads follow their own
specifications instead (domain, speeds, noise); those are checked against
their formulas."""
import math

import numpy as np

from chimera_b200 import problems as P
from oracle.oracle import Config

PI = 3.1415926535897932
TWO_PI = 6.2831853071795865
FOUR_PI = 12.566370614359173


def _grid(n):
    dx = 1.0 / n
    xlin = (np.arange(1, n + 1, dtype=np.float64) - 0.5) * dx
    X = np.ascontiguousarray(np.broadcast_to(xlin[None, :], (n, n)))   # X(ix, iy) = xlin(ix)
    Y = np.ascontiguousarray(np.broadcast_to(xlin[:, None], (n, n)))   # Y(ix, iy) = xlin(iy)
    return dx, xlin, X, Y


def _oracle_cfg(cfg):
    return Config(nx=cfg.nx, ny=cfg.ny, dx=cfg.dx, dy=cfg.dy, gamma=cfg.gamma, bc=cfg.bc)


def _conserved(oracle, cfg, rho, vx, vy, p_thermal, b_x, b_y, Bx=None, By=None):
    c = _oracle_cfg(cfg)
    if Bx is None:
        Bx, By = oracle.average_face_to_cell_B(c, b_x, b_y)
    P_total = p_thermal + 0.5 * (Bx * Bx + By * By)
    M, Mx, My, E = oracle.get_conserved(c, *[np.ascontiguousarray(a) for a in (rho, vx, vy, P_total, Bx, By)])
    return [M, Mx, My, E, b_x, b_y]


def _assert_same(got, want):
    for q, (a, b) in enumerate(zip(got, want)):
        assert np.array_equal(a, b), q


def test_orszag_tang_is_setup_OT_vortex(oracle):
    """src/mhd_init.f90:296-311."""
    n = 48
    cfg, st = P.orszag_tang(n)
    dx, _, X, Y = _grid(n)
    assert cfg.bc == (1, 1, 1, 1) and cfg.dx == dx
    rho = np.full((n, n), 25.0 / (36.0 * PI))
    p = np.full((n, n), 5.0 / (12.0 * PI))
    vx = -np.sin(TWO_PI * Y)
    vy = np.sin(TWO_PI * X)
    Az = np.cos(FOUR_PI * X) / (FOUR_PI * math.sqrt(FOUR_PI)) + np.cos(TWO_PI * Y) / (TWO_PI * math.sqrt(FOUR_PI))
    b_x, b_y = oracle.compute_curl_2d(_oracle_cfg(cfg), np.ascontiguousarray(Az))
    _assert_same(st, _conserved(oracle, cfg, rho, vx, vy, p, b_x, b_y))


def test_field_loop_is_setup_FL_advec(oracle):
    """src/mhd_init.f90:360-391 (unit square, v = (-2, -1))."""
    n = 40
    cfg, st = P.field_loop(n, n, 1.0, 1.0, v=(-2.0, -1.0))
    dx, _, X, Y = _grid(n)
    r0, A0, x0, y0 = 0.3, 1.0e-3, 0.5, 0.5
    r = np.sqrt((X - x0) ** 2 + (Y - y0) ** 2)
    Az = np.where(r < r0, A0 * (r0 - r), 0.0)
    b_x, b_y = oracle.compute_curl_2d(_oracle_cfg(cfg), np.ascontiguousarray(Az))
    ones = np.ones((n, n))
    _assert_same(st, _conserved(oracle, cfg, ones, -2.0 * ones, -1.0 * ones, ones, b_x, b_y))


def test_rotor_is_setup_rotor(oracle):
    """src/mhd_init.f90:399-450, by its per-cell loop."""
    n = 40
    cfg, st = P.rotor(n)
    dx, xlin, _, _ = _grid(n)
    assert cfg.bc == (3, 3, 3, 3) and cfg.gamma == 1.4
    x0 = y0 = 0.5
    r0, r1, u0 = 0.1, 0.115, 2.0
    rho = np.ones((n, n))
    vx = np.zeros((n, n))
    vy = np.zeros((n, n))
    for iy in range(n):
        for ix in range(n):
            rx = float(xlin[ix]) - x0
            ry = float(xlin[iy]) - y0
            r = math.sqrt(rx * rx + ry * ry)
            if r <= r0:
                rho[iy, ix] = 10.0
                vx[iy, ix] = -(u0 * (ry / r0))
                vy[iy, ix] = u0 * (rx / r0)
            elif r < r1:
                f = (r1 - r) / (r1 - r0)
                rho[iy, ix] = 1.0 + 9.0 * f
                if r > 0.0:
                    vx[iy, ix] = -(f * u0 * (ry / r))
                    vy[iy, ix] = f * u0 * (rx / r)
    Bx = np.full((n, n), 5.0 / math.sqrt(4.0 * PI))
    By = np.zeros((n, n))
    b_x, b_y = Bx.copy(), By.copy()             # face B = the uniform cell B
    _assert_same(st, _conserved(oracle, cfg, rho, vx, vy, np.ones((n, n)), b_x, b_y, Bx, By))


def test_kelvin_helmholtz_follows_its_specification(oracle):
    """The Kelvin-Helmholtz workload (not the reference's top-hat set-up):
    [0,1] x [-1,1] periodic, gamma 1.4, HLLD; rho = 1, p = 2.5,
    vx = 0.5 tanh(y'/0.05) with y' mirrored at |y| = 1/2, vy = 0.01 sin(2 pi x)
    exp(-y^2/0.01) + uniform noise of amplitude 1e-3 (seeded), Bx = 0.1."""
    n = 64
    cfg, st = P.kelvin_helmholtz(n)
    assert (cfg.dx, cfg.dy, cfg.gamma, cfg.riemann, cfg.bc) == (1.0 / n, 2.0 / n, 1.4, 3, (1, 1, 1, 1))
    rho, vx, vy, Ptot, Bx, By = oracle.primitives(cfg, st)
    x = (np.arange(1, n + 1) - 0.5) / n
    y = -1.0 + (np.arange(1, n + 1) - 0.5) * 2.0 / n
    X, Y = np.meshgrid(x, y)
    ym = np.where(Y > 0.5, 1.0 - Y, np.where(Y < -0.5, -1.0 - Y, Y))
    assert np.array_equal(rho, np.ones((n, n)))
    assert np.max(np.abs(Bx - 0.1)) == 0.0 and np.max(np.abs(By)) == 0.0
    assert np.max(np.abs((Ptot - 0.5 * (Bx * Bx + By * By)) - 2.5)) < 1e-13
    assert np.max(np.abs(vx - 0.5 * np.tanh(ym / 0.05))) < 1e-15
    noise = vy - 0.01 * np.sin(2.0 * np.pi * X) * np.exp(-Y * Y / 0.01)
    assert np.max(np.abs(noise)) <= 1e-3 * (1 + 1e-12)
    assert 0.5e-3 < noise.std() < 0.65e-3 and abs(noise.mean()) < 1e-4
    assert np.array_equal(P.kelvin_helmholtz(n)[1][2], st[2])            # seeded
    assert not np.array_equal(P.kelvin_helmholtz(n, seed=1)[1][2], st[2])


def test_adjoint_field_loop_follows_its_specification(oracle):
    """The adjoint workload's field loop: [0,2] x [0,1] periodic, v = (2, 1),
    HLLE + Van Leer, gamma 5/3, rho = p = 1, A_z = 1e-3 (0.3 - r) about
    (1, 0.5), so |B| = 1e-3 inside the loop away from its centre and rim."""
    cfg, st = P.field_loop(128, 64)
    assert (cfg.dx, cfg.dy, cfg.gamma, cfg.riemann, cfg.limiter) == (2.0 / 128, 1.0 / 64, 5.0 / 3.0, 2, 1)
    rho, vx, vy, Ptot, Bx, By = oracle.primitives(cfg, st)
    assert np.array_equal(rho, np.ones_like(rho))
    assert np.max(np.abs(vx - 2.0)) < 1e-14 and np.max(np.abs(vy - 1.0)) < 1e-14
    x = (np.arange(1, 129) - 0.5) * cfg.dx
    y = (np.arange(1, 65) - 0.5) * cfg.dy
    X, Y = np.meshgrid(x, y)
    r = np.sqrt((X - 1.0) ** 2 + (Y - 0.5) ** 2)
    B = np.sqrt(Bx * Bx + By * By)
    ring = (r > 0.06) & (r < 0.24)
    assert np.max(np.abs(B[ring] - 1e-3)) < 5e-5
    assert np.max(B[r > 0.33]) == 0.0
    d = oracle.compute_divB(_oracle_cfg(cfg), st[4], st[5])
    assert np.max(np.abs(d)) < 1e-15


def test_grf_members_follow_their_specification(oracle):
    """GRF ensemble members: periodic unit square, rho = p = 1, gamma in
    [1.4, 5/3], face-centred B from a smoothed A_z with rms |B| in [0.2, 1],
    divergence free; velocity with rms |v| in [0.5, 2] before the cap step,
    which scales the velocities alone by 3 / max(c_f + |v|) where that maximum
    exceeds 3 (src/mhd_init.f90:811-829)."""
    n = 64
    capped = 0
    for seed in range(8):
        cfg, st = P.grf_member(n, 1000 + seed)
        _, raw = P.grf_member(n, 1000 + seed, cf_cap=1e30)
        assert 1.4 <= cfg.gamma <= 5.0 / 3.0 and cfg.bc == (1, 1, 1, 1) and cfg.dx == 1.0 / n
        rho, vx, vy, Ptot, Bx, By = oracle.primitives(cfg, st)
        _, ux, uy, _, _, _ = oracle.primitives(cfg, raw)
        B2 = Bx * Bx + By * By
        assert np.max(np.abs(rho - 1.0)) < 1e-15
        assert np.max(np.abs((Ptot - 0.5 * B2) - 1.0)) < 1e-12
        assert 0.2 - 1e-12 <= math.sqrt(float(np.mean(B2))) <= 1.0 + 1e-12
        assert 0.5 - 1e-12 <= math.sqrt(float(np.mean(ux * ux + uy * uy))) <= 2.0 + 1e-12
        assert np.array_equal(st[4], raw[4]) and np.array_equal(st[5], raw[5])     # B never rescaled
        top = float(np.max(np.sqrt(cfg.gamma + B2) + np.sqrt(ux * ux + uy * uy)))
        if top > 3.0:
            capped += 1
            nz = np.abs(ux) > 1e-8
            assert np.max(np.abs(vx[nz] / ux[nz] - 3.0 / top)) < 1e-12
        else:
            assert np.array_equal(st[1], raw[1]) and np.array_equal(st[2], raw[2])
        d = oracle.compute_divB(_oracle_cfg(cfg), st[4], st[5])
        assert np.max(np.abs(d)) < 1e-12
    assert 0 < capped < 8          # both branches of the cap step seen
