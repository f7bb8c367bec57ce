"""Edge cases on the GPU, in place of a sanitizer (compute-sanitizer is closed on
this pool):

* tiny and thin grids (4 x 4 up to 16 x 4, smaller than a tile, so that one
  tile's halo wraps the grid more than once, or clamps on both sides) against
  the oracle bit for bit, for every solver, boundary mix and tile variant;
* canary padding around every array the library writes -- pitched state
  arrays on the host and the device, the packed ghost rows, the per-routine
  outputs and the caller arrays of the no-allocation step -- must come back
  untouched, and the inputs must not change.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from chimera_b200 import ops
from chimera_b200 import problems as P
from chimera_b200.config import BC_OUTFLOW, BC_PERIODIC, HLLD, HLLE, MC, RUSANOV, VAN_LEER, SolverConfig
from tests.gpu_util import max_ulp, require_gpu

pytestmark = pytest.mark.gpu

CANARY = -1.2345678901234567e300


@pytest.fixture(scope="module")
def G():
    return require_gpu()


def _state(nx, ny, bc, seed, riemann=HLLE, limiter=MC, gamma=5.0 / 3.0):
    """A rough seeded state (MOOD and floors active) on an nx x ny grid."""
    rng = np.random.default_rng(seed)
    dx, dy = 1.0 / nx, 1.0 / ny
    px, py = bc[0] == BC_PERIODIC, bc[2] == BC_PERIODIC
    rho = 1.0 + 0.5 * rng.random((ny, nx))
    vx = rng.random((ny, nx)) - 0.5
    vy = rng.random((ny, nx)) - 0.5
    p = 0.5 + rng.random((ny, nx))
    Az = 0.05 * rng.random((ny, nx))
    b_x, b_y = P.curl_2d(Az, dx, dy, px, py)
    Bx, By = P.face_to_cell(b_x, b_y, px, py)
    M, Mx, My, E = P.get_conserved(rho, vx, vy, p + 0.5 * (Bx * Bx + By * By), Bx, By, gamma, dx * dy)
    cfg = SolverConfig(nx=nx, ny=ny, dx=dx, dy=dy, gamma=gamma, riemann=riemann, limiter=limiter, bc=bc)
    return cfg, [np.ascontiguousarray(a) for a in (M, Mx, My, E, b_x, b_y)]


PER = (BC_PERIODIC,) * 4
OUT = (BC_OUTFLOW,) * 4
MIX = (BC_PERIODIC, BC_PERIODIC, BC_OUTFLOW, BC_OUTFLOW)
XOUT = (BC_OUTFLOW, BC_OUTFLOW, BC_PERIODIC, BC_PERIODIC)
TINY = {
    "4x4_periodic": (4, 4, PER),
    "4x4_outflow": (4, 4, OUT),
    "8x8_periodic": (8, 8, PER),
    "4x16_periodic": (4, 16, PER),
    "16x4_outflow": (16, 4, OUT),
    "5x7_mixed": (5, 7, MIX),
    "7x5_xoutflow": (7, 5, XOUT),
}


@pytest.mark.parametrize("solver", [RUSANOV, HLLE, HLLD])
@pytest.mark.parametrize("case", sorted(TINY))
def test_tiny_grids_bitwise_every_variant(G, oracle, case, solver):
    nx, ny, bc = TINY[case]
    cfg, st = _state(nx, ny, bc, seed=nx * 31 + ny, riemann=solver,
                     limiter=VAN_LEER if solver == HLLD else MC)
    ref = oracle.State(st)
    oracle.run(cfg, ref, 6)
    s = G.Solver(cfg)
    for v in range(s.variant_count()):
        s.set_state(st)
        s.set_time(0.0, 1)
        s.set_variant(v)
        s.step(6)
        out = s.get_state()
        for q in range(6):
            assert np.array_equal(out[q], ref.a[q]), (case, v, q, max_ulp(out[q], ref.a[q]))
        assert s.diag()["status"] == 0
    s.close()


def test_canaries_around_pitched_state_arrays(G):
    """set / get / step_host with a leading dimension beyond nx, on host and
    device arrays: the padding columns and the row after the last keep their
    canary, and the inputs are not written."""
    cfg, st = P.orszag_tang(40)
    nx = ny = 40
    ld = 53
    host_in = []
    for a in st:
        b = np.full((ny + 1, ld), CANARY)
        b[:ny, :nx] = a
        host_in.append(b)
    host_in_copy = [b.copy() for b in host_in]
    s = G.Solver(cfg)
    s.set_state([b[:ny, :nx] for b in host_in])
    s.step(2)
    host_out = [np.full((ny + 1, ld), CANARY) for _ in range(6)]
    s.get_state(out=[b[:ny, :nx] for b in host_out])
    dev_out = [torch.full((ny + 1, ld), CANARY, dtype=torch.float64, device="cuda") for _ in range(6)]
    s.get_state(out=[t[:ny, :nx] for t in dev_out])
    ref = G.Solver(cfg)
    ref.set_state(st)
    ref.step(2)
    want = ref.get_state()
    for q in range(6):
        assert np.array_equal(host_in[q], host_in_copy[q])
        for b in (host_out[q], dev_out[q].cpu().numpy()):
            assert np.array_equal(b[:ny, :nx], want[q])
            assert np.all(b[:ny, nx:] == CANARY) and np.all(b[ny, :] == CANARY)
    s.close()
    ref.close()
    # one step on host arrays with the same pitch (chimera_step_host), from t = 0
    s = G.Solver(cfg)
    hin = [b.copy() for b in host_in]
    hout = [np.full((ny + 1, ld), CANARY) for _ in range(6)]
    s.step_host([b[:ny, :nx] for b in hin], out=[b[:ny, :nx] for b in hout])
    ref = G.Solver(cfg)
    ref.set_state(st)
    ref.step(1)
    want = ref.get_state()
    for q in range(6):
        assert np.array_equal(hin[q], host_in[q])
        assert np.array_equal(hout[q][:ny, :nx], want[q])
        assert np.all(hout[q][:ny, nx:] == CANARY) and np.all(hout[q][ny, :] == CANARY)
    s.close()
    ref.close()


def test_canaries_after_packed_ghost_rows(G):
    cfg, st = P.orszag_tang(32)
    s = G.Solver(cfg)
    s.set_state(st)
    rows, n = 4, 6 * 4 * 32
    lo = torch.full((n + 129,), CANARY, dtype=torch.float64, device="cuda")
    hi = torch.full((n + 129,), CANARY, dtype=torch.float64, device="cuda")
    s.halo_pack(rows, lo[:n], hi[:n])
    torch.cuda.synchronize()
    assert torch.all(lo[n:] == CANARY) and torch.all(hi[n:] == CANARY)
    assert not torch.any(lo[:n] == CANARY)
    s.close()


def _bufs(n, k, pad=131):
    """k output buffers of n doubles, each followed by `pad` canary doubles."""
    return [torch.full((n + pad,), CANARY, dtype=torch.float64, device="cuda") for _ in range(k)]


def _p(t):
    return C.c_void_p(t.data_ptr())


def _clean(bufs, n):
    torch.cuda.synchronize()
    return all(bool(torch.all(b[n:] == CANARY)) for b in bufs)


def test_canaries_around_routine_outputs(G):
    """Every per-routine entry point writes exactly its output arrays."""
    cfg, st = _state(24, 18, MIX, seed=5)
    nx, ny = cfg.nx, cfg.ny
    n, npad = nx * ny, (nx + 2) * (ny + 2)
    dev = [torch.from_numpy(a).cuda() for a in st]
    ins_before = [t.clone() for t in dev]
    M, Mx, My, E, bx, by = dev

    B = _bufs(n, 2)
    ops._call("chimera_op_average_face_to_cell_B", cfg, _p(bx), _p(by), *[_p(b) for b in B])
    assert _clean(B, n)
    Bx, By = B[0][:n].view(ny, nx).clone(), B[1][:n].view(ny, nx).clone()

    prim = _bufs(n, 4)
    ops._call("chimera_op_get_primitive", cfg, _p(M), _p(Mx), _p(My), _p(E), _p(Bx), _p(By),
              *[_p(b) for b in prim])
    assert _clean(prim, n)
    rho, vx, vy, Pt = [b[:n].view(ny, nx).clone() for b in prim]

    cons = _bufs(n, 4)
    ops._call("chimera_op_get_conserved", cfg, _p(rho), _p(vx), _p(vy), _p(Pt), _p(Bx), _p(By),
              *[_p(b) for b in cons])
    assert _clean(cons, n)

    pad = _bufs(npad, 1)
    ops._call("chimera_op_fill_ghost_cells", cfg, _p(rho), _p(pad[0]))
    assert _clean(pad, npad)
    rho_pad = pad[0][:npad].view(ny + 2, nx + 2).clone()

    for name in ("chimera_op_compute_gradients", "chimera_op_apply_slope_limiter"):
        g = _bufs(n, 2)
        ops._call(name, cfg, _p(rho_pad), *[_p(b) for b in g])
        assert _clean(g, n), name
    fdx, fdy = g[0][:n].view(ny, nx).clone(), g[1][:n].view(ny, nx).clone()

    rec = _bufs(n, 4)
    ops._call("chimera_op_reconstruction", cfg, _p(rho), _p(fdx), _p(fdy), *[_p(b) for b in rec], C.c_int(1))
    assert _clean(rec, n)

    states = [rho, rho, vx, vx, vy, vy, Pt, Pt, Bx, Bx, By, By]
    fl = _bufs(n, 5)
    ops._call("chimera_op_compute_fluxes", cfg, (C.c_void_p * 12)(*[t.data_ptr() for t in states]),
              (C.c_void_p * 5)(*[b.data_ptr() for b in fl]))
    assert _clean(fl, n)
    fx = fl[4][:n].view(ny, nx).clone()

    F = _bufs(n, 1)
    F[0][:n] = M.reshape(-1)
    ops._call("chimera_op_update_conserved", cfg, _p(F[0]), _p(fx), _p(fx), C.c_double(1e-3))
    assert _clean(F, n)

    bxy = _bufs(n, 3)
    bxy[0][:n] = bx.reshape(-1)
    bxy[1][:n] = by.reshape(-1)
    ops._call("chimera_op_constrained_transport", cfg, _p(bxy[0]), _p(bxy[1]), _p(fx), _p(fx),
              C.c_double(1e-3), _p(bxy[2]))
    assert _clean(bxy, n)

    curl = _bufs(n, 2)
    ops._call("chimera_op_compute_curl_2d", cfg, _p(rho), *[_p(b) for b in curl])
    assert _clean(curl, n)

    d = _bufs(n, 1)
    ops._call("chimera_op_compute_divB", cfg, _p(bx), _p(by), _p(d[0]))
    assert _clean(d, n)

    for a, b in zip(dev, ins_before):
        assert torch.equal(a, b)


def test_canaries_around_no_alloc_arrays(G):
    """The no-allocation step (chimera_rk3_step_noalloc) updates the caller's
    six dense arrays in place and nothing after them."""
    f = G.lib().chimera_rk3_step_noalloc
    f.argtypes = [C.POINTER(G.CCfg)] + [C.c_void_p] * 6 + [C.POINTER(C.c_double), C.POINTER(C.c_int),
                                                          C.POINTER(C.c_double), C.c_void_p]
    f.restype = C.c_int
    cfg, st = _state(40, 24, OUT, seed=9)
    n = cfg.nx * cfg.ny
    bufs = _bufs(n, 6)
    for b, a in zip(bufs, st):
        b[:n] = torch.from_numpy(a.reshape(-1)).cuda()
    t, oc, dtn = C.c_double(0.0), C.c_int(1), C.c_double(0.0)
    ccfg = G.to_ccfg(cfg)
    torch.cuda.synchronize()
    for _ in range(2):
        rc = f(C.byref(ccfg), *[_p(b) for b in bufs], C.byref(t), C.byref(oc), C.byref(dtn), None)
        assert rc == 0
    assert _clean(bufs, n)
    ref = G.Solver(cfg)
    ref.set_state(st)
    ref.step(2)
    for b, w in zip(bufs, ref.get_state()):
        assert np.array_equal(b[:n].cpu().numpy().reshape(cfg.ny, cfg.nx), w)
    ref.close()


@pytest.mark.parametrize("case", ["4x4_periodic", "16x4_outflow", "5x7_mixed", "7x5_xoutflow"])
def test_tiny_grids_fp32_every_variant(G, oracle, case):
    """The FP32-bulk kernels (TMA variants included: their tiles fall back to
    plain loads on grids smaller than a box) on tiny grids, against the FP64
    oracle, with MOOD off: on these rough states the MC limiter often
    saturates at exactly a neighbour's value, where the MOOD bound test is a
    coin toss between two precisions (a single flip moves a 35-cell L1 by
    1e-3).  Without MOOD, Rusanov + MC is continuous in the state (rounding
    the start to FP32 moves the FP64 result by about 1e-8 here), so an L1
    bound of 1e-5 per field after 6 steps separates FP32 arithmetic from an
    indexing fault.  The MOOD indexing on tiny grids is checked bitwise in FP64
    above."""
    from chimera_b200.config import FP32_BULK
    from tests.gpu_util import l1_rel
    nx, ny, bc = TINY[case]
    cfg, st = _state(nx, ny, bc, seed=nx * 17 + ny, riemann=RUSANOV)
    cfg = cfg.replace(mood=False)
    ref = oracle.State(st)
    oracle.run(cfg, ref, 6)
    s = G.Solver(cfg.replace(precision=FP32_BULK))
    for v in range(s.variant_count()):
        s.set_state(st)
        s.set_time(0.0, 1)
        s.set_variant(v)
        s.step(6)
        out = s.get_state()
        for q in range(6):
            err = l1_rel(out[q], ref.a[q])
            assert err <= 1e-5, (case, v, q, err)
        assert s.diag()["status"] == 0
    s.close()
