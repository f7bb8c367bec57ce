"""Vectorised PyTorch FP64 restatement of CHIMERA's per-step hot path.

TEST INFRASTRUCTURE ONLY (oracle #2).  It is written independently of
``chimera_oracle.c`` -- whole-array tensor expressions with shifted views, the
way the Fortran source is written -- so the two restatements check each other;
on the same input they must agree bit for bit.  Being differentiable, it is
also the autodiff reference for the hand-written adjoint.

Arrays are ``(ny, nx)`` tensors (x fastest).  Every function names the
reference routine it follows; expression order follows the Fortran so no
rounding differs.
"""
from __future__ import annotations

import numpy as np
import torch

BC_PERIODIC = 1
RUSANOV, HLLE, HLLD = 1, 2, 3
VAN_LEER, MC = 1, 2
P_FLOOR = 1.0e-12
RHO_FLOOR = 1.0e-12
E_FLOOR_FRAC = 1.0e-10


class _IeeeSqrt(torch.autograd.Function):
    """Correctly rounded square root.  PyTorch's vectorised CPU float64 sqrt is
    not correctly rounded (about 1% of inputs are 1 ulp off), while the
    Fortran, C and CUDA paths all use the IEEE operation; the forward value is
    taken from numpy (IEEE) and the derivative is 1/(2 sqrt x)."""

    @staticmethod
    def forward(ctx, x):
        y = torch.from_numpy(np.sqrt(x.detach().cpu().numpy())).to(x.device)
        ctx.save_for_backward(y)
        return y

    @staticmethod
    def backward(ctx, g):
        (y,) = ctx.saved_tensors
        return g * (0.5 / y)


def _sqrt(x):
    return _IeeeSqrt.apply(x)


def _px(cfg):  # x periodic? (both sides must agree on this path)
    return cfg.bc[0] == BC_PERIODIC


def _py(cfg):
    return cfg.bc[2] == BC_PERIODIC


def _cat_x(a, b):
    return torch.cat([a, b], dim=1)


def _cat_y(a, b):
    return torch.cat([a, b], dim=0)


# src/mhd_field_ops.f90:120-156
def average_face_to_cell_B(cfg, b_x, b_y):
    first = 0.5 * (b_x[:, :1] + b_x[:, -1:]) if cfg.bc[0] == BC_PERIODIC else b_x[:, :1]
    Bx = _cat_x(first, 0.5 * (b_x[:, 1:] + b_x[:, :-1]))
    firsty = 0.5 * (b_y[:1, :] + b_y[-1:, :]) if cfg.bc[2] == BC_PERIODIC else b_y[:1, :]
    By = _cat_y(firsty, 0.5 * (b_y[1:, :] + b_y[:-1, :]))
    return Bx, By


# src/mhd_change_states.f90:61-113
def get_primitive(cfg, M, Mx, My, E, Bx, By):
    vol = cfg.dx * cfg.dy
    g = cfg.gamma
    rho = torch.clamp(M / vol, min=RHO_FLOOR)
    vx = Mx / (rho * vol)
    vy = My / (rho * vol)
    halfB2 = 0.5 * (Bx * Bx + By * By)
    P = ((E / vol - 0.5 * rho * (vx * vx + vy * vy)) - halfB2) * (g - 1.0) + halfB2
    P = torch.clamp(P, min=P_FLOOR)
    P = torch.maximum(P, halfB2 + E_FLOOR_FRAC * (0.5 * rho * (vx * vx + vy * vy) + halfB2))
    return rho, vx, vy, P


# src/mhd_change_states.f90:116-166
def apply_conserved_floors(cfg, M, Mx, My, E, Bx, By):
    vol = cfg.dx * cfg.dy
    g = cfg.gamma
    halfB2 = 0.5 * (Bx * Bx + By * By)
    low = M < RHO_FLOOR * vol
    Mx = torch.where(low, torch.zeros_like(Mx), Mx)
    My = torch.where(low, torch.zeros_like(My), My)
    M = torch.where(low, torch.full_like(M, RHO_FLOOR * vol), M)
    E = torch.where(low, torch.maximum(E, (P_FLOOR / (g - 1.0) + halfB2) * vol), E)
    mag = _sqrt(Mx * Mx + My * My)
    v_mag = mag / M
    fast = v_mag > 50.0
    scale = 50.0 * M / torch.where(fast, mag, torch.ones_like(mag))
    Mx = torch.where(fast, Mx * scale, Mx)
    My = torch.where(fast, My * scale, My)
    return M, Mx, My, E


# src/mhd_bc.f90:36-170 (zero-gradient for every non-periodic side)
def fill_ghost_cells(cfg, f):
    ny, nx = f.shape
    left = f[:, -1:] if cfg.bc[0] == BC_PERIODIC else f[:, :1]
    right = f[:, :1] if cfg.bc[1] == BC_PERIODIC else f[:, -1:]
    mid = torch.cat([left, f, right], dim=1)
    bot = f[-1:, :] if cfg.bc[2] == BC_PERIODIC else f[:1, :]
    top = f[:1, :] if cfg.bc[3] == BC_PERIODIC else f[-1:, :]

    def corner(ix, iy, bcx, bcy):  # 0-based nearest interior corner
        ixw, iyw = nx - 1 - ix, ny - 1 - iy
        if bcx == BC_PERIODIC and bcy == BC_PERIODIC:
            return f[iyw:iyw + 1, ixw:ixw + 1]
        if bcx == BC_PERIODIC:
            return f[iy:iy + 1, ixw:ixw + 1]
        if bcy == BC_PERIODIC:
            return f[iyw:iyw + 1, ix:ix + 1]
        return f[iy:iy + 1, ix:ix + 1]

    b = cfg.bc
    brow = torch.cat([corner(0, 0, b[0], b[2]), bot, corner(nx - 1, 0, b[1], b[2])], dim=1)
    trow = torch.cat([corner(0, ny - 1, b[0], b[3]), top, corner(nx - 1, ny - 1, b[1], b[3])], dim=1)
    return torch.cat([brow, mid, trow], dim=0)


class _LimiterKinkConvention(torch.autograd.Function):
    """Forward: the limiter value.  Backward: its derivative, except where a
    one-sided difference is exactly zero (not differentiable there): both zero
    -> (1/2, 1/2), one zero -> 1 w.r.t. the zero one and 0 w.r.t. the other --
    the kink convention the GPU adjoint states."""

    @staticmethod
    def forward(ctx, dfL, dfR, limiter):
        with torch.enable_grad():
            a = dfL.detach().requires_grad_()
            b = dfR.detach().requires_grad_()
            s = _limit_plain(a, b, limiter)
        ga, gb = torch.autograd.grad(s, (a, b), torch.ones_like(s), allow_unused=True)
        ga = torch.zeros_like(a) if ga is None else ga
        gb = torch.zeros_like(b) if gb is None else gb
        zl, zr = dfL == 0.0, dfR == 0.0
        both = zl & zr
        ga = torch.where(both, torch.full_like(ga, 0.5), torch.where(zl, torch.ones_like(ga),
                         torch.where(zr, torch.zeros_like(ga), ga)))
        gb = torch.where(both, torch.full_like(gb, 0.5), torch.where(zr, torch.ones_like(gb),
                         torch.where(zl, torch.zeros_like(gb), gb)))
        ctx.save_for_backward(ga, gb)
        return s.detach()

    @staticmethod
    def backward(ctx, g):
        ga, gb = ctx.saved_tensors
        return g * ga, g * gb, None


KINK_CONVENTION = False   # set by the adjoint tests


def _limit(dfL, dfR, limiter):
    if KINK_CONVENTION and (dfL.requires_grad or dfR.requires_grad):
        return _LimiterKinkConvention.apply(dfL, dfR, limiter)
    return _limit_plain(dfL, dfR, limiter)


# src/mhd_derivatives.f90:50-127
def _limit_plain(dfL, dfR, limiter):
    prod = dfL * dfR
    den = dfL + dfR
    zero = (prod <= 0.0) | (torch.abs(den) < 1e-12)
    if limiter == VAN_LEER:
        safe = torch.where(zero, torch.ones_like(den), den)
        s = (2.0 * prod) / safe
    else:
        s = torch.copysign(torch.ones_like(dfL), dfL) * torch.minimum(
            torch.minimum(2.0 * torch.abs(dfL), 2.0 * torch.abs(dfR)), 0.5 * torch.abs(den))
    return torch.where(zero, torch.zeros_like(s), s)


def apply_slope_limiter(cfg, pad):
    inv_dx = 1.0 / cfg.dx
    inv_dy = 1.0 / cfg.dy
    c = pad[1:-1, 1:-1]
    sx = _limit((c - pad[1:-1, :-2]) * inv_dx, (pad[1:-1, 2:] - c) * inv_dx, cfg.limiter)
    sy = _limit((c - pad[:-2, 1:-1]) * inv_dy, (pad[2:, 1:-1] - c) * inv_dy, cfg.limiter)
    return sx, sy


# src/mhd_derivatives.f90:15-47
def compute_gradients(cfg, pad):
    return ((pad[1:-1, 2:] - pad[1:-1, :-2]) * (1.0 / (2.0 * cfg.dx)),
            (pad[2:, 1:-1] - pad[:-2, 1:-1]) * (1.0 / (2.0 * cfg.dy)))


def _nbr(f, cfg):
    """MOOD stencil neighbours with the index rules of
    src/mhd_derivatives.f90:191-206: (ip1, im1, jp1, jm1) views."""
    ip1 = _cat_x(f[:, 1:], f[:, :1] if cfg.bc[1] == BC_PERIODIC else f[:, -1:])
    im1 = _cat_x(f[:, -1:] if cfg.bc[0] == BC_PERIODIC else f[:, :1], f[:, :-1])
    jp1 = _cat_y(f[1:, :], f[:1, :] if cfg.bc[3] == BC_PERIODIC else f[-1:, :])
    jm1 = _cat_y(f[-1:, :] if cfg.bc[2] == BC_PERIODIC else f[:1, :], f[:-1, :])
    return ip1, im1, jp1, jm1


# src/mhd_derivatives.f90:130-229
def reconstruction(cfg, f, sx, sy, rho_or_p):
    hx = 0.5 * cfg.dx
    hy = 0.5 * cfg.dy
    XL = f + hx * sx
    YL = f + hy * sy
    tx = f - hx * sx
    ty = f - hy * sy
    XR = _cat_x(tx[:, 1:], tx[:, :1] if cfg.bc[1] == BC_PERIODIC else f[:, -1:])
    YR = _cat_y(ty[1:, :], ty[:1, :] if cfg.bc[3] == BC_PERIODIC else f[-1:, :])
    if cfg.mood:
        ip1, im1, jp1, jm1 = _nbr(f, cfg)
        lo = torch.minimum(torch.minimum(torch.minimum(torch.minimum(f, ip1), im1), jp1), jm1)
        hi = torch.maximum(torch.maximum(torch.maximum(torch.maximum(f, ip1), im1), jp1), jm1)
        if rho_or_p:
            lo = torch.clamp(lo, min=0.1e-8)

        def chk(v):
            return torch.where((v < lo) | (v > hi), f, v)
        XL, XR, YL, YR = chk(XL), chk(XR), chk(YL), chk(YR)
    if rho_or_p:
        XL, XR, YL, YR = (torch.clamp(v, min=1.0e-8) for v in (XL, XR, YL, YR))
    return XL, XR, YL, YR


# src/mhd_derivatives.f90:232-293; slot = dict field -> face tensor
def thermal_pressure_check(slot, cell):
    p_th = slot["P"] - 0.5 * (slot["Bx"] ** 2 + slot["By"] ** 2)
    bad = p_th < P_FLOOR
    return {k: torch.where(bad, cell[k], v) for k, v in slot.items()}


# src/mhd_flux.f90:197-288
def rusanov(g, rL, rR, uL, uR, vL, vR, PL, PR, BxL, BxR, ByL, ByR):
    hL = 0.5 * (BxL * BxL + ByL * ByL)
    hR = 0.5 * (BxR * BxR + ByR * ByR)
    pL = torch.clamp(PL - hL, min=P_FLOOR)
    pR = torch.clamp(PR - hR, min=P_FLOOR)
    eL = pL / (g - 1.0) + 0.5 * rL * (uL * uL + vL * vL) + hL
    eR = pR / (g - 1.0) + 0.5 * rR * (uR * uR + vR * vR) + hR
    ra = 0.5 * (rL + rR)
    ir = 1.0 / ra
    mxa = 0.5 * (rL * uL + rR * uR)
    mya = 0.5 * (rL * vL + rR * vR)
    ea = 0.5 * (eL + eR)
    bxa = 0.5 * (BxL + BxR)
    bya = 0.5 * (ByL + ByR)
    Pa = (g - 1.0) * (ea - 0.5 * (mxa * mxa + mya * mya) * ir - 0.5 * (bxa * bxa + bya * bya)) \
        + 0.5 * (bxa * bxa + bya * bya)
    fM = mxa
    fMx = mxa * mxa * ir + Pa - bxa * bxa
    fMy = mxa * mya * ir - bxa * bya
    fE = (ea + Pa) * mxa * ir - bxa * (bxa * mxa + bya * mya) * ir
    fB = (bya * mxa - bxa * mya) * ir
    cL2 = (g * pL + 2.0 * hL) / rL
    cR2 = (g * pR + 2.0 * hR) / rR
    CL = _sqrt(0.5 * (cL2 + torch.abs(cL2))) + torch.abs(uL)
    CR = _sqrt(0.5 * (cR2 + torch.abs(cR2))) + torch.abs(uR)
    Cm = 0.5 * torch.maximum(CL, CR)
    return (fM - Cm * (rR - rL), fMx - Cm * (rR * uR - rL * uL), fMy - Cm * (rR * vR - rL * vL),
            fE - Cm * (eR - eL), fB - Cm * (ByR - ByL))


def _phys(g, r, u, v, PT, Bx, By):
    h = 0.5 * (Bx * Bx + By * By)
    p = torch.clamp(PT - h, min=P_FLOOR)
    e = p / (g - 1.0) + 0.5 * r * (u * u + v * v) + h
    return h, p, e


# src/mhd_flux.f90:291-405
def hlle(g, rL, rR, uL, uR, vL, vR, PL, PR, BxL, BxR, ByL, ByR):
    hL, pL, eL = _phys(g, rL, uL, vL, PL, BxL, ByL)
    hR, pR, eR = _phys(g, rR, uR, vR, PR, BxR, ByR)
    qL = (g * pL + 2.0 * hL) / rL
    qR = (g * pR + 2.0 * hR) / rR
    cL = torch.clamp(_sqrt(0.5 * (qL + torch.abs(qL))), max=100.0)
    cR = torch.clamp(_sqrt(0.5 * (qR + torch.abs(qR))), max=100.0)
    SL = torch.minimum(uL - cL, uR - cR)
    SR = torch.maximum(uL + cL, uR + cR)
    FL = (rL * uL, rL * uL * uL + PL - BxL * BxL, rL * uL * vL - BxL * ByL,
          (eL + PL) * uL - BxL * (BxL * uL + ByL * vL), ByL * uL - BxL * vL)
    FR = (rR * uR, rR * uR * uR + PR - BxR * BxR, rR * uR * vR - BxR * ByR,
          (eR + PR) * uR - BxR * (BxR * uR + ByR * vR), ByR * uR - BxR * vR)
    dU = (rR - rL, rR * uR - rL * uL, rR * vR - rL * vL, eR - eL, ByR - ByL)
    inv = 1.0 / torch.clamp(SR - SL, min=1.0e-12)
    out = []
    for fl, fr, du in zip(FL, FR, dU):
        f = (SR * fl - SL * fr + SL * SR * du) * inv
        f = torch.where(SL >= 0.0, fl, f)
        f = torch.where(SR <= 0.0, fr, f)
        out.append(f)
    return tuple(out)


# src/mhd_flux.f90:408-779 (branches evaluated everywhere, then selected)
def hlld(g, rL, rR, uL, uR, vL, vR, PL, PR, BxL, BxR, ByL, ByR):
    one = torch.ones_like(rL)
    hL, pL, eL = _phys(g, rL, uL, vL, PL, BxL, ByL)
    hR, pR, eR = _phys(g, rR, uR, vR, PR, BxR, ByR)
    vdL = uL * BxL + vL * ByL
    vdR = uR * BxR + vR * ByR
    FL = (rL * uL, rL * (uL * uL) + PL - BxL * BxL, rL * uL * vL - BxL * ByL,
          (eL + PL) * uL - BxL * vdL, ByL * uL - BxL * vL)
    FR = (rR * uR, rR * (uR * uR) + PR - BxR * BxR, rR * uR * vR - BxR * ByR,
          (eR + PR) * uR - BxR * vdR, ByR * uR - BxR * vR)
    caL = (BxL * BxL) / rL
    caR = (BxR * BxR) / rR
    csL = g * pL / rL
    csR = g * pR / rR
    b2L = (BxL * BxL + ByL * ByL) / rL
    b2R = (BxR * BxR + ByR * ByR) / rR
    tL = csL + b2L
    tR = csR + b2R
    cfL = torch.clamp(_sqrt(0.5 * (tL + _sqrt(torch.clamp(tL * tL - 4.0 * csL * caL, min=0.0)))), max=50.0)
    cfR = torch.clamp(_sqrt(0.5 * (tR + _sqrt(torch.clamp(tR * tR - 4.0 * csR * caR, min=0.0)))), max=50.0)
    SL = torch.minimum(uL - cfL, uR - cfR)
    SR = torch.maximum(uL + cfL, uR + cfR)
    dU = (rR - rL, rR * uR - rL * uL, rR * vR - rL * vL, eR - eL, ByR - ByL)
    dS = SR - SL
    dS_safe = torch.where(dS == 0.0, one, dS)
    inv = 1.0 / dS_safe
    HLL = tuple((SR * fl - SL * fr + SL * SR * du) * inv for fl, fr, du in zip(FL, FR, dU))

    den = rR * (SR - uR) - rL * (SL - uL)
    den = torch.where(torch.abs(den) < 1.0e-15, torch.copysign(torch.full_like(den, 1.0e-15), den), den)
    SM = (rR * uR * (SR - uR) - rL * uL * (SL - uL) - (PR - PL)) / den
    pTs = PL + rL * (SL - uL) * (SM - uL)
    use_hll2 = (SM <= SL + 1.0e-6 * (SR - SL)) | (SM >= SR - 1.0e-6 * (SR - SL))
    pTs = torch.clamp(pTs, min=P_FLOOR)
    dLm = torch.where(SL - SM == 0.0, one, SL - SM)
    dRm = torch.where(SR - SM == 0.0, one, SR - SM)

    def star(r, u, v, e, PT, Bx, By, S, dSm, vd):
        rs = r * (S - u) / dSm
        dd = r * (S - u) * (S - SM) - Bx * Bx
        ok = torch.abs(dd) > 1.0e-3 * torch.maximum(torch.maximum(torch.abs(r * (S - u) * (S - SM)), Bx * Bx),
                                                   torch.full_like(dd, 1.0e-30))
        dds = torch.where(ok, dd, one)
        vs = torch.where(ok, v - Bx * By * (SM - u) / dds, v)
        bs = torch.where(ok, By * (r * ((S - u) * (S - u)) - Bx * Bx) / dds, By)
        vds = SM * Bx + vs * bs
        es = (e * (S - u) - PT * u + pTs * SM + Bx * (vd - vds)) / dSm
        return rs, vs, bs, vds, es

    rLs, vLs, bLs, vdLs, eLs = star(rL, uL, vL, eL, PL, BxL, ByL, SL, dLm, vdL)
    rRs, vRs, bRs, vdRs, eRs = star(rR, uR, vR, eR, PR, BxR, ByR, SR, dRm, vdR)
    sqL = _sqrt(torch.clamp(rLs, min=RHO_FLOOR))
    sqR = _sqrt(torch.clamp(rRs, min=RHO_FLOOR))
    bxa = 0.5 * (BxL + BxR)
    SLs = SM - torch.abs(bxa) / sqL
    SRs = SM + torch.abs(bxa) / sqR
    gen = torch.abs(bxa) > 1.0e-10
    sg = torch.copysign(one, bxa)
    dss = sqL + sqR
    vss = torch.where(gen, (sqL * vLs + sqR * vRs + sg * (bRs - bLs)) / dss, 0.5 * (vLs + vRs))
    bss = torch.where(gen, (sqL * bRs + sqR * bLs + sg * sqL * sqR * (vRs - vLs)) / dss, 0.5 * (bLs + bRs))
    vdss = SM * bxa + vss * bss
    eLss = torch.where(gen, eLs - sqL * sg * (vdLs - vdss), eLs)
    eRss = torch.where(gen, eRs + sqR * sg * (vdRs - vdss), eRs)
    SLs = torch.where(gen, SLs, SM)
    SRs = torch.where(gen, SRs, SM)

    L2 = (FL[0] + SL * (rLs - rL), FL[1] + SL * (rLs * SM - rL * uL), FL[2] + SL * (rLs * vLs - rL * vL),
          FL[3] + SL * (eLs - eL), FL[4] + SL * (bLs - ByL))
    L3 = (L2[0], L2[1], L2[2] + SLs * rLs * (vss - vLs), L2[3] + SLs * (eLss - eLs), L2[4] + SLs * (bss - bLs))
    R2 = (FR[0] + SR * (rRs - rR), FR[1] + SR * (rRs * SM - rR * uR), FR[2] + SR * (rRs * vRs - rR * vR),
          FR[3] + SR * (eRs - eR), FR[4] + SR * (bRs - ByR))
    R3 = (R2[0], R2[1], R2[2] + SRs * rRs * (vss - vRs), R2[3] + SRs * (eRss - eRs), R2[4] + SRs * (bss - bRs))
    left = SM >= 0.0
    F = tuple(torch.where(left, torch.where(SLs >= 0.0, a, b), torch.where(SRs <= 0.0, c, d))
              for a, b, c, d in zip(L2, L3, R2, R3))
    Smax = torch.maximum(torch.abs(SL), torch.abs(SR))
    bnd = (torch.maximum(torch.abs(FL[0]), torch.abs(FR[0])) + Smax * (rL + rR),
           torch.maximum(torch.abs(FL[1]), torch.abs(FR[1])) + Smax * (torch.abs(rL * uL) + torch.abs(rR * uR)),
           torch.maximum(torch.abs(FL[2]), torch.abs(FR[2])) + Smax * (torch.abs(rL * vL) + torch.abs(rR * vR)),
           torch.maximum(torch.abs(FL[3]), torch.abs(FR[3])) + Smax * (torch.abs(eL) + torch.abs(eR)),
           torch.maximum(torch.abs(FL[4]), torch.abs(FR[4])) + Smax * (torch.abs(ByL) + torch.abs(ByR)))
    bad = torch.zeros_like(left)
    for f, b in zip(F, bnd):
        bad = bad | ~torch.isfinite(f) | (torch.abs(f) > 8.0 * b)
    F = tuple(torch.where(bad, h, f) for f, h in zip(F, HLL))
    F = tuple(torch.where(use_hll2, h, f) for f, h in zip(F, HLL))
    F = tuple(torch.where(SR <= 0.0, fr, f) for f, fr in zip(F, FR))
    F = tuple(torch.where(SL >= 0.0, fl, f) for f, fl in zip(F, FL))
    catch1 = (cfL >= 50.0) | (cfR >= 50.0)
    up = tuple(torch.where(cfL <= cfR, fl, fr) for fl, fr in zip(FL, FR))
    return tuple(torch.where(catch1, u, f) for f, u in zip(F, up))


SOLVERS = {RUSANOV: rusanov, HLLE: hlle, HLLD: hlld}


# src/main.f90:346-403
def compute_stage_fluxes(cfg, prim):
    names = ("rho", "vx", "vy", "P", "Bx", "By")
    faces = {}
    for n in names:
        pad = fill_ghost_cells(cfg, prim[n])
        if cfg.slope_limiting:
            sx, sy = apply_slope_limiter(cfg, pad)
        else:
            sx, sy = compute_gradients(cfg, pad)
        faces[n] = reconstruction(cfg, prim[n], sx, sy, n in ("rho", "P"))
    slots = []
    for s in range(4):
        slots.append(thermal_pressure_check({n: faces[n][s] for n in names}, prim))
    XL, XR, YL, YR = slots
    sol = SOLVERS[cfg.riemann]
    fx = sol(cfg.gamma, XL["rho"], XR["rho"], XL["vx"], XR["vx"], XL["vy"], XR["vy"], XL["P"], XR["P"],
             XL["Bx"], XR["Bx"], XL["By"], XR["By"])
    fy = sol(cfg.gamma, YL["rho"], YR["rho"], YL["vy"], YR["vy"], YL["vx"], YR["vx"], YL["P"], YR["P"],
             YL["By"], YR["By"], YL["Bx"], YR["Bx"])
    # x: mass, momx, momy, energy, By ; y (rotated): mass, momy, momx, energy, Bx
    return list(fx), [fy[0], fy[2], fy[1], fy[3], fy[4]]


# src/mhd_flux.f90:20-76
def update_conserved(cfg, F, fX, fY, dt):
    ax = dt * cfg.dy
    ay = dt * cfg.dx
    inx = _cat_x(fX[:, -1:] if cfg.bc[0] == BC_PERIODIC else None, fX[:, :-1]) if cfg.bc[0] == BC_PERIODIC \
        else None
    if cfg.bc[0] == BC_PERIODIC:
        F = F - ax * fX + ax * inx
    else:
        F = _cat_x(F[:, :1] - ax * fX[:, :1], F[:, 1:] - ax * fX[:, 1:] + ax * fX[:, :-1])
    if cfg.bc[2] == BC_PERIODIC:
        iny = _cat_y(fY[-1:, :], fY[:-1, :])
        F = F - ay * fY + ay * iny
    else:
        F = _cat_y(F[:1, :] - ay * fY[:1, :], F[1:, :] - ay * fY[1:, :] + ay * fY[:-1, :])
    return F


# src/mhd_field_ops.f90:15-57
def compute_curl_2d(cfg, Az):
    ix = 1.0 / cfg.dx
    iy = 1.0 / cfg.dy
    bx_in = (Az[1:, :] - Az[:-1, :]) * iy
    bx0 = (Az[:1, :] - Az[-1:, :]) * iy if cfg.bc[2] == BC_PERIODIC else bx_in[:1, :]
    by_in = -((Az[:, 1:] - Az[:, :-1]) * ix)
    by0 = -((Az[:, :1] - Az[:, -1:]) * ix) if cfg.bc[0] == BC_PERIODIC else by_in[:, :1]
    return _cat_y(bx0, bx_in), _cat_x(by0, by_in)


# src/mhd_flux.f90:79-136
def constrained_transport(cfg, bx, by, fByX, fBxY, dt):
    up = _cat_y(fByX[1:, :], fByX[:1, :] if cfg.bc[3] == BC_PERIODIC else fByX[-1:, :])
    right = _cat_x(fBxY[:, 1:], fBxY[:, :1] if cfg.bc[1] == BC_PERIODIC else fBxY[:, -1:])
    Ez = 0.25 * (-fByX - up + fBxY + right)
    dbx, dby = compute_curl_2d(cfg, -Ez)
    return bx + dt * dbx, by + dt * dby


# src/main.f90:118-148
def outflow_correction(cfg, U, prim, dt):
    M, Mx, My, E, bx, by = U
    g = cfg.gamma
    if cfg.bc[0] != BC_PERIODIC:
        r, u, v, P, Bx, By = (prim[k][:, :1] for k in ("rho", "vx", "vy", "P", "Bx", "By"))
        a = dt * cfg.dy
        h = 0.5 * (Bx * Bx + By * By)
        e = (P - h) / (g - 1.0) + 0.5 * r * (u * u + v * v) + h
        M = _cat_x(M[:, :1] + a * r * u, M[:, 1:])
        Mx = _cat_x(Mx[:, :1] + a * (r * (u * u) + P - Bx * Bx), Mx[:, 1:])
        My = _cat_x(My[:, :1] + a * (r * u * v - Bx * By), My[:, 1:])
        E = _cat_x(E[:, :1] + a * ((e + P) * u - Bx * (Bx * u + By * v)), E[:, 1:])
    if cfg.bc[2] != BC_PERIODIC:
        r, u, v, P, Bx, By = (prim[k][:1, :] for k in ("rho", "vx", "vy", "P", "Bx", "By"))
        a = dt * cfg.dx
        h = 0.5 * (Bx * Bx + By * By)
        e = (P - h) / (g - 1.0) + 0.5 * r * (u * u + v * v) + h
        M = _cat_y(M[:1, :] + a * r * v, M[1:, :])
        My = _cat_y(My[:1, :] + a * (r * (v * v) + P - By * By), My[1:, :])
        Mx = _cat_y(Mx[:1, :] + a * (r * v * u - By * Bx), Mx[1:, :])
        E = _cat_y(E[:1, :] + a * ((e + P) * v - By * (By * v + Bx * u)), E[1:, :])
    return [M, Mx, My, E, bx, by]


def primitives(cfg, U):
    Bx, By = average_face_to_cell_B(cfg, U[4], U[5])
    rho, vx, vy, P = get_primitive(cfg, U[0], U[1], U[2], U[3], Bx, By)
    return {"rho": rho, "vx": vx, "vy": vy, "P": P, "Bx": Bx, "By": By}


def stage(cfg, k, U, U0, dt):
    """One RK3 stage (src/main.f90:107-208 / 261-267)."""
    prim = primitives(cfg, U)
    fX, fY = compute_stage_fluxes(cfg, prim)
    M, Mx, My, E = (update_conserved(cfg, U[q], fX[q], fY[q], dt) for q in range(4))
    M, Mx, My, E = apply_conserved_floors(cfg, M, Mx, My, E, prim["Bx"], prim["By"])
    bx, by = constrained_transport(cfg, U[4], U[5], fX[4], fY[4], dt)
    out = outflow_correction(cfg, [M, Mx, My, E, bx, by], prim, dt)
    if k == 2:
        out = [0.75 * a + 0.25 * b for a, b in zip(U0, out)]
    elif k == 3:
        out = [(1.0 / 3.0) * a + (2.0 / 3.0) * b for a, b in zip(U0, out)]
    if k >= 2:
        out[:4] = apply_conserved_floors(cfg, *out[:4], prim["Bx"], prim["By"])
    return out


# src/main.f90:72-83
def cfl_dt(cfg, U, t=0.0, output_count=1):
    p = primitives(cfg, U)
    inv = 1.0 / p["rho"]
    B2 = p["Bx"] * p["Bx"] + p["By"] * p["By"]
    c0 = cfg.gamma * (p["P"] - 0.5 * B2) * inv
    ca = B2 * inv
    cf = _sqrt(c0 + ca)
    cf = torch.where(p["rho"] < 1.0e-3, torch.clamp(cf, max=50.0), cf)
    q = torch.full_like(cf, min(cfg.dx, cfg.dy)) / (cf + _sqrt(p["vx"] * p["vx"] + p["vy"] * p["vy"]))
    dt = cfg.courant * float(q.min())
    if t + dt > output_count * cfg.t_out:
        dt = output_count * cfg.t_out - t
    return max(dt, float(torch.tensor(1e-12, dtype=torch.float32).double()))


def rk3_step(cfg, U, dt):
    """One SSP-RK3 step with a given dt (differentiable in U)."""
    U0 = list(U)
    U1 = stage(cfg, 1, U0, U0, dt)
    U2 = stage(cfg, 2, U1, U0, dt)
    return stage(cfg, 3, U2, U0, dt)
