"""Initial states generated on the device.

The five problems of ``problems`` (set-ups of src/mhd_init.f90:259-860 and of
the workload specifications) built directly in HBM as CUDA float64 tensors:
the primitive fields with torch element-wise operations, then face B from A_z,
cell-centred B and the conserved variables with the reference-routine kernels
(``chimera_op_compute_curl_2d``, ``chimera_op_average_face_to_cell_B``,
``chimera_op_get_conserved``).  The Gaussian random fields are white noise
from a CUDA Philox generator smoothed by a Gaussian RBF in Fourier space
(batched cuFFT over all members of one size), replacing the reference's
O(N^4) direct DFT (src/mhd_init.f90:686-701).

Results: (cfg, [Mass, Momx, Momy, Energy, b_x, b_y]) like ``problems``; the
analytic problems agree with the host generators to rounding, the random ones
have the same statistics from a device random stream (not the host stream's
numbers).
"""
from __future__ import annotations

import math

import torch

from . import ops
from . import problems as P
from .config import BC_OUTFLOW, BC_PERIODIC, FP64, HLLD, HLLE, MC, RUSANOV, VAN_LEER, SolverConfig

_F64 = torch.float64


def _centres(n, lo, d):
    return (torch.arange(1, n + 1, dtype=_F64, device="cuda") - 0.5) * d + lo


def _mesh(cfg, lo_x=0.0, lo_y=0.0):
    x = _centres(cfg.nx, lo_x, cfg.dx)
    y = _centres(cfg.ny, lo_y, cfg.dy)
    return x[None, :].expand(cfg.ny, cfg.nx), y[:, None].expand(cfg.ny, cfg.nx)


def _finish(cfg, rho, vx, vy, p_thermal, b_x, b_y):
    """Cell B, total pressure and conserved variables (src/mhd_change_states.f90:16-58)."""
    c = cfg.replace(precision=FP64)
    b_x, b_y = b_x.contiguous(), b_y.contiguous()
    Bx, By = ops.average_face_to_cell_B(c, b_x, b_y)
    Ptot = p_thermal + 0.5 * (Bx * Bx + By * By)
    M, Mx, My, E = ops.get_conserved(c, *(t.contiguous() for t in (rho, vx, vy, Ptot)), Bx, By)
    return [M, Mx, My, E, b_x, b_y]


def _curl(cfg, Az):
    return ops.compute_curl_2d(cfg.replace(precision=FP64), Az.contiguous())


def orszag_tang(n=256, riemann=RUSANOV, limiter=MC, mood=True, t_end=0.5):
    """Orszag-Tang vortex (src/mhd_init.f90:296-311) on the device."""
    dx = 1.0 / n
    cfg = SolverConfig(nx=n, ny=n, dx=dx, dy=dx, gamma=5.0 / 3.0, riemann=riemann, limiter=limiter,
                       mood=mood, t_end=t_end, bc=(BC_PERIODIC,) * 4)
    X, Y = _mesh(cfg)
    two_pi, four_pi = 2.0 * math.pi, 4.0 * math.pi
    Az = torch.cos(four_pi * X) / (four_pi * math.sqrt(four_pi)) + \
        torch.cos(two_pi * Y) / (two_pi * math.sqrt(four_pi))
    b_x, b_y = _curl(cfg, Az)
    full = lambda v: torch.full((n, n), v, dtype=_F64, device="cuda")   # noqa: E731
    return cfg, _finish(cfg, full(25.0 / (36.0 * math.pi)), -torch.sin(two_pi * Y), torch.sin(two_pi * X),
                        full(5.0 / (12.0 * math.pi)), b_x, b_y)


def rotor(n=1024, riemann=HLLE, limiter=MC, mood=True, t_end=0.15):
    """MHD rotor (src/mhd_init.f90:399-450) on the device, outflow sides."""
    dx = 1.0 / n
    cfg = SolverConfig(nx=n, ny=n, dx=dx, dy=dx, gamma=1.4, riemann=riemann, limiter=limiter,
                       mood=mood, t_end=t_end, bc=(BC_OUTFLOW,) * 4)
    X, Y = _mesh(cfg)
    r0, r1, u0 = 0.1, 0.115, 2.0
    rx, ry = X - 0.5, Y - 0.5
    r = torch.sqrt(rx * rx + ry * ry)
    core = r <= r0
    taper = (~core) & (r < r1)
    f = (r1 - r) / (r1 - r0)
    safe_r = torch.where(r > 0, r, torch.ones_like(r))
    rho = torch.where(core, torch.full_like(r, 10.0), torch.where(taper, 1.0 + 9.0 * f, torch.ones_like(r)))
    vx = torch.where(core, -u0 * (ry / r0), torch.where(taper & (r > 0), -f * u0 * (ry / safe_r), torch.zeros_like(r)))
    vy = torch.where(core, u0 * (rx / r0), torch.where(taper & (r > 0), f * u0 * (rx / safe_r), torch.zeros_like(r)))
    b_x = torch.full_like(r, 5.0 / math.sqrt(4.0 * math.pi))
    return cfg, _finish(cfg, rho, vx, vy, torch.ones_like(r), b_x, torch.zeros_like(r))


def field_loop(nx=512, ny=512, lx=2.0, ly=1.0, v=(2.0, 1.0), riemann=HLLE, limiter=VAN_LEER, mood=True,
               t_end=1.0):
    """Field-loop advection (src/mhd_init.f90:360-391 generalised) on the device."""
    cfg = SolverConfig(nx=nx, ny=ny, dx=lx / nx, dy=ly / ny, gamma=5.0 / 3.0, riemann=riemann,
                       limiter=limiter, mood=mood, t_end=t_end, bc=(BC_PERIODIC,) * 4)
    X, Y = _mesh(cfg)
    r = torch.sqrt((X - 0.5 * lx) ** 2 + (Y - 0.5 * ly) ** 2)
    Az = torch.where(r < 0.3, 1.0e-3 * (0.3 - r), torch.zeros_like(r))
    b_x, b_y = _curl(cfg, Az)
    one = torch.ones_like(r)
    return cfg, _finish(cfg, one, torch.full_like(r, float(v[0])), torch.full_like(r, float(v[1])), one, b_x, b_y)


def kelvin_helmholtz(n=4096, riemann=HLLD, limiter=MC, mood=True, seed=0, t_end=1e30):
    """Magnetised Kelvin-Helmholtz of the workload (problems.kelvin_helmholtz)
    on the device; the 1e-3 seed noise comes from the device generator."""
    cfg = SolverConfig(nx=n, ny=n, dx=1.0 / n, dy=2.0 / n, gamma=1.4, riemann=riemann, limiter=limiter,
                       mood=mood, t_end=t_end, bc=(BC_PERIODIC,) * 4)
    X, Y = _mesh(cfg, 0.0, -1.0)
    ym = torch.where(Y > 0.5, 1.0 - Y, torch.where(Y < -0.5, -1.0 - Y, Y))
    gen = torch.Generator(device="cuda").manual_seed(seed)
    noise = torch.rand((n, n), generator=gen, dtype=_F64, device="cuda") * 2.0 - 1.0
    vx = 0.5 * torch.tanh(ym / 0.05)
    vy = 0.01 * torch.sin(2.0 * math.pi * X) * torch.exp(-Y * Y / 0.01) + 1.0e-3 * noise
    one = torch.ones_like(X)
    return cfg, _finish(cfg, one, vx, vy, torch.full_like(X, 2.5), torch.full_like(X, 0.1), torch.zeros_like(X))


def _rbf_smooth(noise, length, d):
    """Periodic convolution of white noise (..., n, n) with exp(-r^2 / (2 l^2)), batched cuFFT."""
    n = noise.shape[-1]
    k = 2.0 * math.pi * torch.fft.fftfreq(n, d=d, dtype=_F64, device="cuda")
    k2 = k[:, None] ** 2 + k[None, :] ** 2
    return torch.fft.ifft2(torch.fft.fft2(noise) * torch.exp(-0.5 * length * length * k2)).real


def grf_parameters(seed):
    """(gamma, V0, B0) of the GRF member seeded with `seed`: the first three
    uniforms of its device stream, gamma ~ U[1.4, 5/3], V0 ~ U[0.5, 2],
    B0 ~ U[0.2, 1]."""
    gen = torch.Generator(device="cuda").manual_seed(int(seed))
    u = torch.rand(3, generator=gen, dtype=_F64, device="cuda").cpu()
    return (1.4 + (5.0 / 3.0 - 1.4) * float(u[0]), 0.5 + 1.5 * float(u[1]), 0.2 + 0.8 * float(u[2]))


def grf_members(n, seeds, length=0.1, cf_cap=3.0):
    """GRF members of one size n (problems.grf_member's specification) on the
    device, one batched FFT for all of them; member k is drawn from a CUDA
    Philox stream seeded with seeds[k]."""
    m = len(seeds)
    params = torch.empty((m, 3), dtype=_F64)
    noise = torch.empty((m, 2, n, n), dtype=_F64, device="cuda")
    for k, seed in enumerate(seeds):
        gen = torch.Generator(device="cuda").manual_seed(int(seed))
        u = torch.rand(3, generator=gen, dtype=_F64, device="cuda").cpu()   # = grf_parameters(seed)
        params[k] = torch.stack([1.4 + (5.0 / 3.0 - 1.4) * u[0], 0.5 + 1.5 * u[1], 0.2 + 0.8 * u[2]])
        noise[k] = torch.randn((2, n, n), generator=gen, dtype=_F64, device="cuda")
    dx = 1.0 / n
    smooth = _rbf_smooth(noise, length, dx)
    psi, Az = smooth[:, 0], smooth[:, 1]
    vx = (torch.roll(psi, -1, dims=1) - torch.roll(psi, 1, dims=1)) / (2.0 * dx)
    vy = -(torch.roll(psi, -1, dims=2) - torch.roll(psi, 1, dims=2)) / (2.0 * dx)
    out = []
    for k in range(m):
        gamma, V0, B0 = (float(x) for x in params[k])
        cfg = SolverConfig(nx=n, ny=n, dx=dx, dy=dx, gamma=gamma, riemann=RUSANOV, limiter=MC, mood=True,
                           t_end=1e30, bc=(BC_PERIODIC,) * 4)
        c = cfg.replace(precision=FP64)
        vrms = torch.sqrt(torch.mean(vx[k] * vx[k] + vy[k] * vy[k]))
        vxk, vyk = vx[k] * (V0 / vrms), vy[k] * (V0 / vrms)
        b_x, b_y = _curl(cfg, Az[k])
        Bx, By = ops.average_face_to_cell_B(c, b_x, b_y)
        scale = B0 / torch.sqrt(torch.mean(Bx * Bx + By * By))
        b_x, b_y = b_x * scale, b_y * scale
        Bx, By = Bx * scale, By * scale
        cf = torch.sqrt(gamma + (Bx * Bx + By * By))            # rho = p = 1
        top = torch.max(cf + torch.sqrt(vxk * vxk + vyk * vyk))
        shrink = torch.clamp(cf_cap / top, max=1.0)              # the cap of src/mhd_init.f90:815-831
        one = torch.ones_like(vxk)
        out.append((cfg, _finish(cfg, one, vxk * shrink, vyk * shrink, one, b_x, b_y)))
    return out


def grf_ensemble(scale=1, precision=FP64, seed0=1000):
    """The GRF ensemble (sizes of problems.grf_ensemble_sizes) on the device:
    member k seeded with seed0 + k.  Returns (cfgs, states)."""
    sizes = P.grf_ensemble_sizes(scale)
    cfgs, states = [None] * len(sizes), [None] * len(sizes)
    for n in sorted(set(sizes)):
        idx = [k for k, s in enumerate(sizes) if s == n]
        for k, (cfg, st) in zip(idx, grf_members(n, [seed0 + k for k in idx])):
            cfgs[k], states[k] = cfg.replace(precision=precision), st
    return cfgs, states


__all__ = ["orszag_tang", "rotor", "field_loop", "kelvin_helmholtz", "grf_parameters", "grf_members",
           "grf_ensemble"]
