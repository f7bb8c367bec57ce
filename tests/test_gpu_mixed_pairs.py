"""A periodic side facing a non-periodic one (a "mixed pair").

The reference fills each side's ghost cells on its own (src/mhd_bc.f90:45-100),
so with x = 0 periodic and x = N outflow the flux entering cell 1 is the
outflow face N+1/2, whose right state is cell N itself; with x = 0 outflow
and x = N periodic the face N+1/2 takes cell 1's reconstruction with the slope
of its outflow ghost (src/mhd_derivatives.f90:148-161, 189-206).  The FP64
handles run such grids through their own kernel instantiation and must match
the FP64 oracle bit for bit, like every other boundary mix (the adjoint's
tests hold their own cases); the FP32 forms, through their own
instantiations, stay within their stated bar of it; the no-allocation step
refuses them.
"""
import numpy as np
import pytest

from chimera_b200 import problems as P
from chimera_b200.config import (BC_FIXED, BC_INFLOW, BC_OUTFLOW, BC_PERIODIC, FP32_BULK, FP32_MIXED, HLLD, HLLE,
                                 RUSANOV, VAN_LEER)
from tests.gpu_util import l1_rel, max_ulp, require_gpu

pytestmark = pytest.mark.gpu

PER, OUT = BC_PERIODIC, BC_OUTFLOW


def _ot(n, bc, **kw):
    cfg, st = P.orszag_tang(n, **kw)
    return cfg.replace(bc=bc), st


def _rotor(n, bc, **kw):
    cfg, st = P.rotor(n, **kw)
    return cfg.replace(bc=bc), st


def _ragged(bc):
    cfg, st = P.field_loop(50, 37, 1.0, 37.0 / 50.0, riemann=HLLD)
    return cfg.replace(bc=bc), st


CASES = {
    "xlo_periodic_hlle_mc": (lambda: _ot(48, (PER, OUT, PER, PER), riemann=HLLE), 30),
    "xhi_periodic_hlld_vl": (lambda: _ot(48, (OUT, PER, OUT, OUT), riemann=HLLD, limiter=VAN_LEER), 30),
    "ylo_periodic_rusanov": (lambda: _ot(48, (PER, PER, PER, OUT), riemann=RUSANOV), 30),
    "yhi_periodic_rotor_hlle": (lambda: _rotor(96, (OUT, OUT, OUT, PER)), 30),
    "both_pairs_rotor_hlld": (lambda: _rotor(96, (PER, OUT, OUT, PER), riemann=HLLD), 25),
    "both_pairs_ragged": (lambda: _ragged((OUT, PER, PER, OUT)), 25),
    "no_slope_limiting": (lambda: (_ot(48, (OUT, PER, PER, OUT))[0].replace(slope_limiting=False),
                                   _ot(48, (OUT, PER, PER, OUT))[1]), 20),
    # a grid smaller than one tile: halo positions wrap more than once
    "tiny_8x6": (lambda: _small(8, 6, (PER, OUT, OUT, PER)), 20),
    # fixed and inflow sides act as outflow (src/main.f90:349-354)
    "fixed_inflow_sides": (lambda: _ot(40, (PER, BC_FIXED, BC_INFLOW, PER), riemann=HLLE), 20),
}


def _small(nx, ny, bc):
    cfg, st = P.field_loop(nx, ny, 1.0, ny / nx, riemann=HLLE)
    return cfg.replace(bc=bc), st


@pytest.fixture(scope="module")
def G():
    return require_gpu()


@pytest.mark.parametrize("case", sorted(CASES))
def test_mixed_pair_bitwise(G, oracle, case):
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
        assert np.array_equal(out[q], ref.a[q]), (case, q, max_ulp(out[q], ref.a[q]))
    assert d["t"] == ref.t and d["output_count"] == ref.output_count
    s.close()


def test_mixed_pair_member_in_a_batch(G, oracle):
    """A batch holding one mixed-pair member runs every member through the
    mixed-pair kernels; each member still equals its oracle run."""
    mem = [_ot(40, (PER,) * 4, riemann=HLLE), _rotor(64, (PER, OUT, OUT, OUT)), _ot(37, (OUT,) * 4, riemann=HLLE)]
    s = G.Solver([c for c, _ in mem])
    assert s.variant_count() == 1
    for m, (_, st) in enumerate(mem):
        s.set_state(st, member=m)
    s.step(10)
    for m, (cfg, st) in enumerate(mem):
        ref = oracle.State(st)
        oracle.run(cfg, ref, 10)
        out = s.get_state(member=m)
        for q in range(6):
            assert np.array_equal(out[q], ref.a[q]), (m, q)
    s.close()


def test_mixed_pair_step_host(G, oracle):
    """chimera_step_host: a mixed y pair takes the whole-grid stages (no
    wavefront over row chunks); a mixed x pair keeps the wavefront."""
    for bc in ((PER, PER, OUT, PER), (PER, OUT, OUT, OUT)):
        cfg, st = _rotor(64, bc)
        ref = oracle.State(st)
        oracle.run(cfg, ref, 2)
        s = G.Solver(cfg)
        out = s.step_host(st)
        out = s.step_host(out)
        for q in range(6):
            assert np.array_equal(out[q], ref.a[q]), (bc, q)
        s.close()


@pytest.mark.parametrize("precision", [FP32_BULK, FP32_MIXED])
@pytest.mark.parametrize("bc", [(PER, OUT, PER, PER), (OUT, PER, OUT, PER), (PER, OUT, OUT, PER)])
def test_reduced_precision_forms_on_mixed_pairs(G, oracle, precision, bc):
    """The FP32 forms run mixed pairs through their own instantiations: within
    the FP32 forms' stated bar of the FP64 oracle (L1 <= 1e-5 per field; Orszag-
    Tang 64^2, HLLE + MC + MOOD, 30 steps)."""
    cfg, st = _ot(64, bc, riemann=HLLE)
    ref = oracle.State(st)
    oracle.run(cfg, ref, 30)
    s = G.Solver(cfg.replace(precision=precision))
    assert s.variant_count() == 1
    s.set_state(st)
    s.step(30)
    out, d = s.get_state(), s.diag()
    s.close()
    errs = [l1_rel(out[q], ref.a[q]) for q in range(6)]
    assert max(errs) <= 1e-5, errs
    assert d["status"] == 0
