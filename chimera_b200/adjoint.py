"""Differentiation of an RK3 run through the hand-written discrete adjoint.

``RK3Run`` is a ``torch.autograd.Function``: forward advances the conserved
state (six CUDA float64 tensors) by ``len(dts)`` SSP-RK3 steps with the given
time steps, keeping a checkpoint every ``K`` steps; backward re-runs each
K-step segment from its checkpoint and applies the adjoint step
(``chimera_adjoint_step``) in reverse.

Conventions (stated): the time steps are frozen -- dt is an input, not a
function of the state, so the derivative of the CFL reduction is not taken;
obtain the dt sequence from a primal run (``cfl_dts``) and reuse it.  The MOOD,
floor and thermal-check decisions and the limiter branches are the forward's;
at a kink the derivative is that of the branch the forward took (one-sided).
Periodic or outflow sides, each side on its own.

Forward precision: FP64 (the tape kernels, bit-identical to the fused FP64
step) or a reduced form -- ``FP32_BULK`` or ``FP32_MIXED`` -- in which the
forward steps run through the fused FP32 solver with the same frozen time
steps (``chimera_set_dt_device`` before each step) and the loss is the
reduced-precision result.  The checkpoints are that forward's states (as FP64);
backward re-runs each segment from its checkpoint in FP64 and applies the FP64
adjoint, so the gradient is the FP64 adjoint along the reduced-precision
trajectory, restarted from it every K steps.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import gpu
from .config import BC_PERIODIC, FP32_BULK, FP32_MIXED, FP64, SolverConfig

_bound = False


def _lib():
    global _bound
    L = gpu.lib()
    if not _bound:
        P = C.c_void_p
        arr6 = P * 6
        L.chimera_adjoint_create.argtypes = [C.POINTER(gpu.CCfg), P, C.POINTER(P)]
        L.chimera_adjoint_step.argtypes = [P, arr6, C.c_double, arr6, arr6]
        L.chimera_adjoint_forward_step.argtypes = [P, arr6, C.c_double, arr6]
        L.chimera_adjoint_destroy.argtypes = [P]
        L.chimera_adjoint_destroy.restype = None
        _bound = True
    return L


def _ptr6(ts):
    for t in ts:
        if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
            raise ValueError("expected contiguous CUDA float64 tensors")
    return (C.c_void_p * 6)(*[t.data_ptr() for t in ts])


class Adjoint:
    """Handle for the adjoint kernels of one grid (FP64; periodic or outflow sides, each on its own)."""

    def __init__(self, cfg: SolverConfig):
        self.cfg = cfg.replace(precision=FP64)
        h = C.c_void_p()
        ccfg = gpu.to_ccfg(self.cfg)
        stream = torch.cuda.current_stream().cuda_stream
        rc = _lib().chimera_adjoint_create(C.byref(ccfg), C.c_void_p(stream), C.byref(h))
        if rc != 0:
            raise gpu.ChimeraError(rc, "chimera_adjoint_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            _lib().chimera_adjoint_destroy(self._h)
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

    def forward_step(self, U, dt):
        out = [torch.empty_like(u) for u in U]
        rc = _lib().chimera_adjoint_forward_step(self._h, _ptr6(U), float(dt), _ptr6(out))
        if rc != 0:
            raise gpu.ChimeraError(rc, "chimera_adjoint_forward_step")
        return out

    def step_vjp(self, U, dt, lam_next):
        lam = [torch.empty_like(u) for u in U]
        rc = _lib().chimera_adjoint_step(self._h, _ptr6(U), float(dt), _ptr6(lam_next), _ptr6(lam))
        if rc != 0:
            raise gpu.ChimeraError(rc, "chimera_adjoint_step")
        return lam


def cfl_dts(cfg: SolverConfig, U, nsteps: int):
    """The dt sequence of an FP64 primal run from U (the CFL dt with the tOut
    clip of every step), through the fused solver."""
    dts = []
    with gpu.Solver(cfg.replace(precision=FP64)) as s:
        s.set_state([u.contiguous() for u in U])
        for _ in range(nsteps):
            dts.append(s.diag()["dt"])
            s.step(1)
    return dts


def _forward_reduced(cfg: SolverConfig, U0, dts, K: int, precision: int):
    """The forward steps in a reduced-precision form with the given time steps:
    (checkpoints every K steps as FP64 tensors, final state as FP64 tensors)."""
    # t_end / t_out far away: every step is taken with the dt given (the CFL
    # dt the solver computes after each step is overwritten before the next)
    c = cfg.replace(precision=precision, t_end=1.0e300, t_out=1.0e300)
    dt_dev = torch.tensor([float(d) for d in dts], dtype=torch.float64, device=U0[0].device)
    torch.cuda.current_stream().synchronize()   # the solver's own stream reads U0 and dt_dev
    checkpoints = [(0, [u.clone() for u in U0])]
    with gpu.Solver(c) as s:
        s.set_state(U0)
        for i in range(len(dts)):
            s.set_dt_device(dt_dev[i:i + 1])
            s.step(1)
            if (i + 1) % K == 0 and i + 1 < len(dts):
                ck = [torch.empty_like(u) for u in U0]
                s.get_state(out=ck)
                checkpoints.append((i + 1, ck))
        final = [torch.empty_like(u) for u in U0]
        s.get_state(out=final)
    return checkpoints, final


class RK3Run(torch.autograd.Function):
    """U_N = RK3^N(U_0) with frozen dts; checkpoints every K steps; forward
    in FP64 or a reduced-precision form (module docstring)."""

    @staticmethod
    def forward(ctx, adj: Adjoint, dts, K: int, precision: int, *U0):
        U = [u.detach().contiguous() for u in U0]
        if precision == FP64:
            checkpoints = [(0, [u.clone() for u in U])]
            for s, dt in enumerate(dts):
                U = adj.forward_step(U, dt)
                if (s + 1) % K == 0 and s + 1 < len(dts):
                    checkpoints.append((s + 1, [u.clone() for u in U]))
        elif precision in (FP32_BULK, FP32_MIXED):
            checkpoints, U = _forward_reduced(adj.cfg, U, dts, K, precision)
        else:
            raise ValueError(f"unknown forward precision {precision}")
        ctx.adj = adj
        ctx.dts = list(dts)
        ctx.K = K
        ctx.checkpoints = checkpoints
        return tuple(U)

    @staticmethod
    def backward(ctx, *grads):
        adj, dts = ctx.adj, ctx.dts
        lam = [g.contiguous() if g is not None else None for g in grads]
        if any(x is None for x in lam):
            ref = next(x for x in lam if x is not None)
            lam = [x if x is not None else torch.zeros_like(ref) for x in lam]
        n = len(dts)
        for k in range(len(ctx.checkpoints) - 1, -1, -1):
            start, U = ctx.checkpoints[k]
            end = ctx.checkpoints[k + 1][0] if k + 1 < len(ctx.checkpoints) else n
            states = [U]
            for s in range(start, end - 1):          # recompute the segment's states
                states.append(adj.forward_step(states[-1], dts[s]))
            for s in range(end - 1, start - 1, -1):
                lam = adj.step_vjp(states[s - start], dts[s], lam)
        return (None, None, None, None, *lam)


def run(adj: Adjoint, U0, dts, K: int = 20, precision: int = FP64):
    """Differentiable RK3 run (see RK3Run); ``precision`` is the forward's
    (FP64, FP32_BULK or FP32_MIXED); the adjoint is FP64."""
    return RK3Run.apply(adj, list(dts), int(K), int(precision), *U0)


# --- helpers for losses on primitive inputs ------------------------------------

def _cell_B(cfg: SolverConfig, b_x, b_y):
    """average_face_to_cell_B (src/mhd_field_ops.f90:120-156): the mean of a
    cell's two faces; at a non-periodic low side the face value itself."""
    Bx = 0.5 * (b_x + torch.roll(b_x, 1, dims=1))
    By = 0.5 * (b_y + torch.roll(b_y, 1, dims=0))
    if cfg.bc[0] != BC_PERIODIC:
        Bx = torch.cat([b_x[:, :1], Bx[:, 1:]], dim=1)
    if cfg.bc[2] != BC_PERIODIC:
        By = torch.cat([b_y[:1, :], By[1:, :]], dim=0)
    return Bx, By


def conserved_from_primitive(cfg: SolverConfig, rho, vx, vy, p_thermal, b_x, b_y):
    """Torch version of get_conserved (src/mhd_change_states.f90:16-58) with the
    cell-centred B of face B, differentiable in every input."""
    Bx, By = _cell_B(cfg, b_x, b_y)
    vol = cfg.dx * cfg.dy
    P = p_thermal + 0.5 * (Bx * Bx + By * By)
    rho_cp = torch.clamp(rho, min=1.0e-12)
    P_cp = torch.clamp(P, min=1.0e-12)
    Mass = rho_cp * vol
    halfB2 = 0.5 * (Bx * Bx + By * By)
    Energy = ((P_cp - halfB2) / (cfg.gamma - 1.0) + 0.5 * rho_cp * (vx * vx + vy * vy) + halfB2) * vol
    return [Mass, Mass * vx, Mass * vy, Energy, b_x, b_y]


def magnetic_energy(cfg: SolverConfig, U):
    """sum 1/2 |B|^2 vol over cells, B cell centred from the faces."""
    Bx, By = _cell_B(cfg, U[4], U[5])
    return 0.5 * torch.sum(Bx * Bx + By * By) * (cfg.dx * cfg.dy)
