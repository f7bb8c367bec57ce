"""The reference's module routines as GPU kernels (chimera_b200.ops):
  * the reference's Fortran known-answer tests (tests/fortran/*.f90, ported in
    tests/test_oracle_kat.py) re-run with the GPU routines in place of the
    oracle;
  * bitwise parity of every routine with the oracle on evolved states, every
    boundary combination (including one periodic side), all three solvers."""
import numpy as np
import pytest
import torch

from chimera_b200 import problems as P
from chimera_b200.config import BC_OUTFLOW, BC_PERIODIC, HLLD, HLLE, MC, RUSANOV, VAN_LEER
from tests import test_oracle_kat as kat
from tests.gpu_util import require_gpu

pytestmark = pytest.mark.gpu


def _d(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def _h(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


class GpuAsOracle:
    """The oracle's numpy-in / numpy-out signatures over the GPU routines."""

    def __init__(self):
        require_gpu()
        from chimera_b200 import ops
        self.ops = ops

    def fill_ghost_cells(self, cfg, f):
        return _h(self.ops.fill_ghost_cells(cfg, _d(f)))

    def get_conserved(self, cfg, *a):
        return tuple(_h(x) for x in self.ops.get_conserved(cfg, *[_d(x) for x in a]))

    def get_primitive(self, cfg, *a):
        return tuple(_h(x) for x in self.ops.get_primitive(cfg, *[_d(x) for x in a]))

    def compute_curl_2d(self, cfg, Az):
        return tuple(_h(x) for x in self.ops.compute_curl_2d(cfg, _d(Az)))

    def compute_divB(self, cfg, bx, by):
        return _h(self.ops.compute_divB(cfg, _d(bx), _d(by)))

    def compute_gradients(self, cfg, pad):
        return tuple(_h(x) for x in self.ops.compute_gradients(cfg, _d(pad)))


@pytest.fixture(scope="module")
def oracle():                      # the Fortran KATs, run on the GPU routines
    return GpuAsOracle()


test_bcs_periodic = kat.test_bcs_periodic
test_bcs_outflow = kat.test_bcs_outflow
test_bcs_mixed = kat.test_bcs_mixed
test_change_states_round_trip = kat.test_change_states_round_trip
test_change_states_density_floor = kat.test_change_states_density_floor
test_change_states_proportional_floor = kat.test_change_states_proportional_floor
test_div_curl_is_zero = kat.test_div_curl_is_zero
test_div_curl_is_zero_nonperiodic = kat.test_div_curl_is_zero_nonperiodic
test_gradient_linear_exact = kat.test_gradient_linear_exact
test_gradient_sinusoid_second_order = kat.test_gradient_sinusoid_second_order


# ---- bitwise parity with the oracle ------------------------------------------
BCS = {
    "periodic": (BC_PERIODIC,) * 4,
    "outflow": (BC_OUTFLOW,) * 4,
    "x_periodic": (BC_PERIODIC, BC_PERIODIC, BC_OUTFLOW, BC_OUTFLOW),
    "one_sided": (BC_PERIODIC, BC_OUTFLOW, BC_OUTFLOW, BC_PERIODIC),
}


@pytest.fixture(scope="module")
def O():
    from oracle import oracle as O
    O.build()
    return O


@pytest.fixture(scope="module")
def ops():
    require_gpu()
    from chimera_b200 import ops
    return ops


def _state(O, bc, riemann=HLLD, limiter=MC, n=40, ny=33, steps=6):
    cfg, st = P.orszag_tang(n, riemann=riemann, limiter=limiter)
    cfg = cfg.replace(bc=(BC_PERIODIC,) * 4)
    s = O.State(st)
    O.run(cfg, s, steps)                        # develop structure first (periodic)
    a = [np.ascontiguousarray(x[:ny, :]) for x in s.a]
    return cfg.replace(ny=ny, bc=bc), a


def _eq(a, b):
    a = a if isinstance(a, np.ndarray) else _h(a)
    assert np.array_equal(a, b), float(np.max(np.abs(a - b)))


@pytest.mark.parametrize("bc", sorted(BCS))
def test_cell_routines_bitwise(O, ops, bc):
    cfg, a = _state(O, BCS[bc])
    Bx, By = O.average_face_to_cell_B(cfg, a[4], a[5])
    gBx, gBy = ops.average_face_to_cell_B(cfg, _d(a[4]), _d(a[5]))
    _eq(gBx, Bx); _eq(gBy, By)
    prim = O.get_primitive(cfg, a[0], a[1], a[2], a[3], Bx, By)
    for x, y in zip(ops.get_primitive(cfg, *[_d(x) for x in (a[0], a[1], a[2], a[3], Bx, By)]), prim):
        _eq(x, y)
    cons = O.get_conserved(cfg, *prim, Bx, By)
    for x, y in zip(ops.get_conserved(cfg, *[_d(x) for x in (*prim, Bx, By)]), cons):
        _eq(x, y)
    # floors: a near-vacuum cell and a fast cell
    M, Mx, My, E = (x.copy() for x in a[:4])
    M[3, 4] = -1.0
    Mx[7, 9] = 1e3 * M[7, 9]
    ref = O.apply_conserved_floors(cfg, M, Mx, My, E, Bx, By)
    got = ops.apply_conserved_floors(cfg, *[_d(x) for x in (M, Mx, My, E, Bx, By)])
    for x, y in zip(got, ref):
        _eq(x, y)
    _eq(ops.compute_divB(cfg, _d(a[4]), _d(a[5])), O.compute_divB(cfg, a[4], a[5]))
    bx, by = O.compute_curl_2d(cfg, a[3])
    gbx, gby = ops.compute_curl_2d(cfg, _d(a[3]))
    _eq(gbx, bx); _eq(gby, by)


@pytest.mark.parametrize("bc", sorted(BCS))
@pytest.mark.parametrize("limiter", [MC, VAN_LEER])
def test_reconstruction_chain_bitwise(O, ops, bc, limiter):
    cfg, a = _state(O, BCS[bc], limiter=limiter)
    Bx, By = O.average_face_to_cell_B(cfg, a[4], a[5])
    rho, vx, vy, Pt = O.get_primitive(cfg, a[0], a[1], a[2], a[3], Bx, By)
    for f, rp in ((rho, True), (vx, False), (Pt, True), (By, False)):
        pad = O.fill_ghost_cells(cfg, f)
        _eq(ops.fill_ghost_cells(cfg, _d(f)), pad)
        for name in ("compute_gradients", "apply_slope_limiter"):
            ref = getattr(O, name)(cfg, pad)
            got = getattr(ops, name)(cfg, _d(pad))
            _eq(got[0], ref[0]); _eq(got[1], ref[1])
        sx, sy = O.apply_slope_limiter(cfg, pad)
        for mood in (True, False):
            c2 = cfg.replace(mood=mood)
            ref = O.reconstruction(c2, f, sx, sy, rp)
            got = ops.reconstruction(c2, _d(f), _d(sx), _d(sy), rp)
            for x, y in zip(got, ref):
                _eq(x, y)


@pytest.mark.parametrize("riemann", [RUSANOV, HLLE, HLLD])
def test_compute_fluxes_bitwise(O, ops, riemann):
    cfg, a = _state(O, BCS["periodic"], riemann=riemann)
    Bx, By = O.average_face_to_cell_B(cfg, a[4], a[5])
    prim = list(O.get_primitive(cfg, a[0], a[1], a[2], a[3], Bx, By)) + [Bx, By]
    faces = []
    for k, f in enumerate(prim):
        sx, sy = O.apply_slope_limiter(cfg, O.fill_ghost_cells(cfg, f))
        faces.append(O.reconstruction(cfg, f, sx, sy, k in (0, 3)))
    rng = np.random.default_rng(riemann)
    # x faces, then strongly perturbed states (degenerate HLLD branches: weak Bx, fast jumps)
    L = [faces[k][0] for k in range(6)]
    R = [faces[k][1] for k in range(6)]
    R2 = [r * (1.0 + 0.5 * rng.standard_normal(r.shape)) for r in R]
    R2[0] = np.abs(R2[0]) + 0.01
    R2[3] = np.abs(R2[3]) + 0.5 * (R2[4] ** 2 + R2[5] ** 2) + 1e-3
    L2 = [l.copy() for l in L]
    L2[4] = L2[4] * (rng.uniform(size=L2[4].shape) < 0.5) * 1e-11   # Bx ~ 0 on half the faces
    for LL, RR in ((L, R), (L2, R2)):
        args = [LL[0], RR[0], LL[1], RR[1], LL[2], RR[2], LL[3], RR[3], LL[4], RR[4], LL[5], RR[5]]
        ref = O.compute_fluxes(cfg, *args)
        got = ops.compute_fluxes(cfg, *[_d(x) for x in args])
        for x, y in zip(got, ref):
            _eq(x, y)


@pytest.mark.parametrize("bc", sorted(BCS))
def test_update_and_ct_bitwise(O, ops, bc):
    cfg, a = _state(O, BCS[bc])
    rng = np.random.default_rng(3)
    fX = rng.standard_normal(a[0].shape)
    fY = rng.standard_normal(a[0].shape)
    _eq(ops.update_conserved(cfg, _d(a[3]), _d(fX), _d(fY), 1.3e-3), O.update_conserved(cfg, a[3], fX, fY, 1.3e-3))
    bx, by = O.constrained_transport(cfg, a[4], a[5], fX, fY, 1.3e-3)
    gbx, gby = ops.constrained_transport(cfg, _d(a[4]), _d(a[5]), _d(fX), _d(fY), 1.3e-3)
    _eq(gbx, bx); _eq(gby, by)


def test_thermal_pressure_check_bitwise(O, ops):
    cfg, a = _state(O, BCS["periodic"])
    Bx, By = O.average_face_to_cell_B(cfg, a[4], a[5])
    rho, vx, vy, Pt = O.get_primitive(cfg, a[0], a[1], a[2], a[3], Bx, By)
    rng = np.random.default_rng(5)
    cell = dict(P=Pt, Bx=Bx, By=By, rho=rho, vx=vx, vy=vy)
    slots = {k: [v * (1.0 + 0.3 * rng.standard_normal(v.shape)) for _ in range(4)] for k, v in cell.items()}
    slots["P"] = [p * (rng.uniform(size=p.shape) < 0.7) for p in slots["P"]]   # some faces with p_th < 0
    ref = {k: [x.copy() for x in v] for k, v in slots.items()}
    O.lib().orc_thermal_pressure_check
    import ctypes as C
    arr = lambda xs: (C.POINTER(C.c_double) * 4)(*[O._p(x) for x in xs])
    O.lib().orc_thermal_pressure_check(C.byref(O._c(cfg)), arr(ref["P"]), arr(ref["Bx"]), arr(ref["By"]),
                                       arr(ref["rho"]), arr(ref["vx"]), arr(ref["vy"]),
                                       *[O._p(cell[k]) for k in ("rho", "vx", "vy", "P", "Bx", "By")])
    dev = {k: [_d(x) for x in v] for k, v in slots.items()}
    ops.thermal_pressure_check(cfg, dev["P"], dev["Bx"], dev["By"], dev["rho"], dev["vx"], dev["vy"],
                               *[_d(cell[k]) for k in ("rho", "vx", "vy", "P", "Bx", "By")])
    for k in slots:
        for x, y in zip(dev[k], ref[k]):
            _eq(x, y)


def test_floor_velocity_cap_sweep(O, ops):
    """The conserved floors' velocity cap (|Mom| / M > 50,
    src/mhd_change_states.f90:116-166) for speeds across its threshold and
    across 40, below which the GPU skips the reference's square root and
    division (an exact pre-test): bit for bit against the oracle, including
    the speeds 40 and 50 themselves and their neighbouring doubles."""
    cfg, a = _state(O, BCS["periodic"])
    ny, nx = a[0].shape
    n = nx * ny
    rng = np.random.default_rng(3)
    special = [40.0, 50.0, np.nextafter(40.0, 0.0), np.nextafter(40.0, 99.0), np.nextafter(50.0, 0.0),
               np.nextafter(50.0, 99.0), 39.999999999, 40.000000001, 49.9999999999, 50.0000000001, 1e3, 0.0]
    speeds = np.concatenate([np.array(special), np.linspace(0.0, 100.0, n - len(special))])
    rng.shuffle(speeds)
    ang = rng.uniform(0.0, 2.0 * np.pi, n)
    M = (0.5 + rng.random(n)) * cfg.dx * cfg.dy
    Mx = (M * speeds * np.cos(ang)).reshape(ny, nx)
    My = (M * speeds * np.sin(ang)).reshape(ny, nx)
    M = M.reshape(ny, nx)
    E = a[3].copy()
    Bx, By = O.average_face_to_cell_B(cfg, a[4], a[5])
    ref = O.apply_conserved_floors(cfg, M, Mx, My, E, Bx, By)
    got = ops.apply_conserved_floors(cfg, *[_d(x) for x in (M, Mx, My, E, Bx, By)])
    for x, y in zip(got, ref):
        _eq(x, y)
    capped = np.sqrt(ref[1] ** 2 + ref[2] ** 2) / ref[0]
    assert np.sum(speeds > 50.0) > 100 and np.all(capped <= 50.0 * (1 + 1e-12))
