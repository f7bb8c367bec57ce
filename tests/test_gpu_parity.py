"""Parity of the plain FP64 GPU path with the FP64 oracle, through the C-ABI.

The FP64 kernels are compiled without multiply-add contraction and follow the
reference's expression order, so the expected result is bit-for-bit equality
with the oracle; the acceptance bar stated for the drop-in is looser: L1
relative error <= 1e-12 per field and max|divB| * dx / max|B| <= 1e-13.
"""
import numpy as np
import pytest

from chimera_b200 import problems as P
from chimera_b200.config import BC_OUTFLOW, BC_PERIODIC, HLLD, HLLE, MC, RUSANOV, VAN_LEER
from tests.gpu_util import l1_rel, max_ulp, require_gpu

pytestmark = pytest.mark.gpu

L1_TOL = 1e-12
DIVB_TOL = 1e-13


def _mixed(n):
    cfg, st = P.orszag_tang(n)
    return cfg.replace(bc=(BC_PERIODIC, BC_PERIODIC, BC_OUTFLOW, BC_OUTFLOW)), st


def _mixed_xout(n):
    cfg, st = P.orszag_tang(n)
    return cfg.replace(bc=(BC_OUTFLOW, BC_FIXED_, BC_PERIODIC, BC_PERIODIC)), st


BC_FIXED_ = 2


CASES = {
    "ot64_rusanov_mc": (lambda: P.orszag_tang(64), 30),
    "ot64_hlle_mc": (lambda: P.orszag_tang(64, riemann=HLLE), 30),
    "ot64_hlld_vl": (lambda: P.orszag_tang(64, riemann=HLLD, limiter=VAN_LEER), 30),
    "rotor96_hlle_mood": (lambda: P.rotor(96), 30),
    "rotor96_hlld_nomood": (lambda: P.rotor(96, riemann=HLLD, mood=False), 30),
    "rotor96_rusanov_vl": (lambda: P.rotor(96, riemann=RUSANOV, limiter=VAN_LEER), 30),
    "field_loop_64x32_hlle_vl": (lambda: P.field_loop(64, 32), 30),
    "kh_48_hlld": (lambda: P.kelvin_helmholtz(48, riemann=HLLD), 30),
    "grf_64": (lambda: P.grf_member(64, 11), 30),
    "mixed_periodic_outflow": (lambda: _mixed(48), 30),
    "mixed_fixed_is_outflow": (lambda: _mixed_xout(48), 20),
    "no_slope_limiting": (lambda: (P.orszag_tang(48)[0].replace(slope_limiting=False), P.orszag_tang(48)[1]), 20),
    "ragged_50x37": (lambda: _ragged(), 25),
}


def _ragged():
    cfg, st = P.field_loop(50, 37, 1.0, 37.0 / 50.0, riemann=HLLD, limiter=MC)
    return cfg, st


@pytest.fixture(scope="module")
def G():
    return require_gpu()


@pytest.mark.parametrize("case", sorted(CASES))
def test_step_parity_bitwise(G, oracle, case):
    make, nsteps = CASES[case]
    cfg, st = make()
    ref = oracle.State(st)
    dts = oracle.run(cfg, ref, nsteps)
    s = G.Solver(cfg)
    s.set_state(st)
    dts_gpu = []
    for _ in range(nsteps):
        dts_gpu.append(s.diag()["dt"])
        s.step(1)
    out = s.get_state()
    d = s.diag()
    assert np.array_equal(np.array(dts_gpu), dts), "dt sequence differs"
    for q in range(6):
        assert l1_rel(out[q], ref.a[q]) <= L1_TOL, (q, l1_rel(out[q], ref.a[q]))
        assert np.array_equal(out[q], ref.a[q]), (case, q, max_ulp(out[q], ref.a[q]))
    assert d["t"] == ref.t
    assert d["output_count"] == ref.output_count
    s.close()


def test_stage_parity(G, oracle):
    """Each RK stage separately against the oracle's stage (src/main.f90:107-267)."""
    cfg, st = P.orszag_tang(64, riemann=HLLE)
    warm = oracle.State(st)
    oracle.run(cfg, warm, 12)   # develop some structure so MOOD and limiters are active
    u0 = warm.a
    dt = 1.7e-3
    s = G.Solver(cfg)
    s.set_state(u0)
    s.stage(1, dt)
    u1 = oracle.stage(cfg, 1, dt, u0, u0)
    g1 = s.get_stage_buffer(1)
    for q in range(6):
        assert np.array_equal(g1[q], u1[q]), ("stage1", q, max_ulp(g1[q], u1[q]))
    s.stage(2, dt)
    u2 = oracle.stage(cfg, 2, dt, u1, u0)
    g2 = s.get_stage_buffer(2)
    for q in range(6):
        assert np.array_equal(g2[q], u2[q]), ("stage2", q, max_ulp(g2[q], u2[q]))
    s.stage(3, dt)
    u3 = oracle.stage(cfg, 3, dt, u2, u0)
    g3 = s.get_state()
    for q in range(6):
        assert np.array_equal(g3[q], u3[q]), ("stage3", q, max_ulp(g3[q], u3[q]))
    s.close()


def test_orszag_tang_256_100_steps(G, oracle):
    """The drop-in gate: OT 256^2, Rusanov + MC (+MOOD), CFL 0.3, 100 steps."""
    cfg, st = P.orszag_tang(256)
    ref = oracle.State(st)
    oracle.run(cfg, ref, 100)
    s = G.Solver(cfg)
    s.set_state(st)
    s.step(100)
    out = s.get_state()
    d = s.diag()
    for q in range(6):
        assert l1_rel(out[q], ref.a[q]) <= L1_TOL
    assert d["divb_rel"] <= DIVB_TOL
    assert d["steps"] == 100
    ndiff = sum(int(np.sum(out[q] != ref.a[q])) for q in range(6))
    assert ndiff == 0, f"{ndiff} values differ from the oracle"


def test_advance_to_t_end(G, oracle):
    """do while (t < tEnd) with the tOut clipping, on the device."""
    cfg, st = P.orszag_tang(48, t_end=0.045)
    ref = oracle.State(st)
    n_ref = len(oracle.run(cfg, ref, 10000))
    s = G.Solver(cfg)
    s.set_state(st)
    n = s.advance()
    d = s.diag()
    assert n == n_ref
    assert d["t"] == ref.t and d["active"] == 0
    out = s.get_state()
    for q in range(6):
        assert np.array_equal(out[q], ref.a[q])


@pytest.mark.parametrize("graph_steps", [0, 5])
def test_advance_output_stops_at_every_output_time(G, oracle, graph_steps):
    """chimera_advance_output: the device-resident loop stops right after each
    step that reaches an output time (src/main.f90:279-292), with the oracle's
    state, t and outputCount there, snapshot after snapshot, and with nothing
    left paused after the last one (t_end)."""
    cfg, st = P.orszag_tang(48, t_end=0.05)
    cfg = cfg.replace(t_out=0.01)
    ref = oracle.State(st)
    s = G.Solver(cfg)
    if graph_steps:
        s.set_graph_steps(graph_steps)
    s.set_state(st)
    snaps = 0
    while s.diag()["active"]:
        oc0 = ref.output_count
        n_ref = 0
        while ref.output_count == oc0 and ref.t < cfg.t_end:   # the reference's loop to its next snapshot
            n_ref += len(oracle.run(cfg, ref, 1))
        n = s.advance_output()
        d = s.diag()
        assert n == n_ref and d["t"] == ref.t and d["output_count"] == ref.output_count
        out = s.get_state()
        for q in range(6):
            assert np.array_equal(out[q], ref.a[q]), (snaps, q)
        snaps += 1
    assert snaps == 5 and d["t"] == ref.t and d["active"] == 0
    assert s.advance_output() == 0            # t >= t_end: nothing more to do
    # a member resumed after its pause steps on with chimera_step
    s.set_time(0.0, 1)
    s.set_state(st)
    s.advance_output()
    t1 = s.diag()["t"]
    s.step(1)
    d = s.diag()
    assert d["t"] > t1 and d["active"] == 1 and d["output_count"] == 2


def test_graph_replay_matches_eager(G):
    cfg, st = P.rotor(64)
    a = G.Solver(cfg)
    a.set_state(st)
    a.step(8)
    b = G.Solver(cfg)
    b.set_state(st)
    b.set_graph_steps(4)
    b.step(4)
    b.step(4)
    for x, y in zip(a.get_state(), b.get_state()):
        assert np.array_equal(x, y)


def test_determinism(G):
    cfg, st = P.orszag_tang(96, riemann=HLLD)
    res = []
    for _ in range(2):
        s = G.Solver(cfg)
        s.set_state(st)
        s.step(10)
        res.append((s.get_state(), s.diag()))
    for x, y in zip(res[0][0], res[1][0]):
        assert np.array_equal(x, y)
    assert res[0][1]["divb_mean"] == res[1][1]["divb_mean"]


def test_diagnostics_match_oracle(G, oracle):
    cfg, st = P.orszag_tang(64)
    ref = oracle.State(st)
    oracle.run(cfg, ref, 5)
    s = G.Solver(cfg)
    s.set_state(st)
    s.step(5)
    d = s.diag()
    div = oracle.compute_divB(cfg, ref.a[4], ref.a[5])
    assert d["divb_max"] == np.max(np.abs(div))
    assert abs(d["divb_mean"] - np.mean(np.abs(div))) <= 1e-12 * max(np.mean(np.abs(div)), 1e-300)
    assert abs(d["mass"] - ref.a[0].sum()) <= 1e-13 * abs(ref.a[0].sum())
    rho, vx, vy, Pt, Bx, By = oracle.primitives(cfg, ref.a)
    assert d["dt"] == oracle.cfl_dt(cfg, rho, vx, vy, Pt, Bx, By, ref.t, ref.output_count)


def test_device_pointers_and_pitch(G):
    """set/get through device memory with a padded leading dimension."""
    import torch
    cfg, st = P.orszag_tang(40)
    ld = 48
    dev = []
    for a in st:
        t = torch.zeros((40, ld), dtype=torch.float64, device="cuda")
        t[:, :40] = torch.from_numpy(a)
        dev.append(t[:, :40])
    s = G.Solver(cfg)
    s.set_state(dev)
    s.step(3)
    outd = [torch.zeros((40, ld), dtype=torch.float64, device="cuda")[:, :40] for _ in range(6)]
    s.get_state(out=outd)
    h = G.Solver(cfg)
    h.set_state(st)
    h.step(3)
    for x, y in zip(outd, h.get_state()):
        assert np.array_equal(x.cpu().numpy(), y)


def test_rotor_1024_full_size(G, oracle):
    """The rotor workload at full size (1024^2, outflow, HLLE + MC + MOOD)."""
    cfg, st = P.rotor(1024)
    ref = oracle.State(st)
    oracle.set_omp_mode(2)
    try:
        oracle.run(cfg, ref, 4)
    finally:
        oracle.set_omp_mode(0)
    s = G.Solver(cfg)
    s.set_state(st)
    s.step(4)
    out = s.get_state()
    for q in range(6):
        assert np.array_equal(out[q], ref.a[q]), q
    assert s.diag()["divb_rel"] <= DIVB_TOL


@pytest.mark.parametrize("solver", [RUSANOV, HLLE, HLLD])
def test_every_tile_variant_bitwise(G, oracle, solver):
    """Every compiled tile shape / occupancy variant gives the same bits."""
    cfg, st = P.orszag_tang(70, riemann=solver)
    cfg = cfg.replace(bc=(BC_PERIODIC, BC_PERIODIC, BC_OUTFLOW, BC_OUTFLOW))
    ref = oracle.State(st)
    oracle.run(cfg, ref, 8)
    s = G.Solver(cfg)
    for v in range(s.variant_count()):
        s.set_state(st)
        s.set_time(0.0, 1)
        s.set_variant(v)
        s.step(8)
        out = s.get_state()
        bad = [q for q in range(6) if not np.array_equal(out[q], ref.a[q])]
        if bad:
            # report the size of the difference and whether a fresh handle
            # reproduces it, then fail
            q = bad[0]
            t = G.Solver(cfg)
            t.set_variant(v)
            t.set_state(st)
            t.step(8)
            again = t.get_state()
            t.close()
            fresh_ok = all(np.array_equal(again[k], ref.a[k]) for k in range(6))
            pytest.fail(f"variant {v} {s.variant()}: fields {bad} differ from the oracle, field {q}: "
                        f"{int(np.sum(out[q] != ref.a[q]))} cells, max {max_ulp(out[q], ref.a[q])} ulp; "
                        f"a fresh handle of this variant matches the oracle: {fresh_ok}")


def test_tma_and_plain_loads_in_one_batch(G, oracle):
    """The default variant loads interior tiles by TMA where the member has
    tensor maps; a member whose row pitch is not a multiple of 16 bytes (odd
    nx) has none and takes the plain loads everywhere.  A batch holding both,
    and the odd grid alone, match the oracle bit for bit."""
    members = [P.orszag_tang(96, riemann=HLLE), P.field_loop(101, 64, 101.0 / 64.0, 1.0, riemann=HLLE, limiter=MC)]
    cfgs = [c for c, _ in members]
    s = G.Solver(cfgs)
    s.set_variant(0)
    for m, (_, st) in enumerate(members):
        s.set_state(st, member=m)
    s.step(6)
    for m, (cfg, st) in enumerate(members):
        ref = oracle.State(st)
        oracle.run(cfg, ref, 6)
        out = s.get_state(member=m)
        for q in range(6):
            assert np.array_equal(out[q], ref.a[q]), (m, q)
    s.close()


def test_autotune_keeps_state(G, oracle):
    """Autotuning runs dry steps only: state and time-loop counters unchanged."""
    cfg, st = P.rotor(128)
    s = G.Solver(cfg)
    s.set_state(st)
    s.step(2)
    before, d0 = s.get_state(), s.diag()
    v, ms = s.autotune(reps=2)
    assert 0 <= v < s.variant_count() and ms > 0
    after, d1 = s.get_state(), s.diag()
    for x, y in zip(before, after):
        assert np.array_equal(x, y)
    assert (d0["t"], d0["steps"], d0["dt"]) == (d1["t"], d1["steps"], d1["dt"])
    s.step(3)
    ref = oracle.State(st)
    oracle.run(cfg, ref, 5)
    for x, y in zip(s.get_state(), ref.a):
        assert np.array_equal(x, y)
