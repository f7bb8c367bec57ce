"""Solver switches and constants.

The numbering of every switch is the reference's code numbering
(``src/mhd_config.f90:27-43``), not the README's table: BC_FIXED = 2 and
BC_OUTFLOW = 3 (the README swaps the two).  FIXED and INFLOW behave as
zero-gradient outflow on this path because the time loop never passes an
ambient state to ``fill_ghost_cells`` (``src/main.f90:349-354``).
"""
from __future__ import annotations

from dataclasses import dataclass, field

# src/mhd_config.f90:33-36
RUSANOV, HLLE, HLLD = 1, 2, 3
# src/mhd_config.f90:28-29
VAN_LEER, MC = 1, 2
# src/mhd_config.f90:40-43
BC_PERIODIC, BC_FIXED, BC_OUTFLOW, BC_INFLOW = 1, 2, 3, 4

# precision forms of the GPU path
FP64 = 0        # plain FP64, bit-compatible with the FP64 restatement
FP32_BULK = 1   # FP32 storage and bulk arithmetic; FP64 pressure recovery, dt and sums
FP32_MIXED = 2  # FP64 storage; FP32 reconstruction / limiter / MOOD / Riemann arithmetic; FP64 pressure
                # recovery, updates, floors, RK blends, dt and sums


@dataclass
class SolverConfig:
    """One grid's configuration.  Defaults are the reference's build-time
    parameters (src/mhd_config.f90:16-62)."""
    nx: int
    ny: int
    dx: float
    dy: float
    gamma: float
    courant: float = 0.3          # courant_fac
    t_out: float = 0.01           # tOut
    t_end: float = 1.0            # tEnd
    bc: tuple = field(default_factory=lambda: (BC_PERIODIC,) * 4)  # xlo, xhi, ylo, yhi
    riemann: int = RUSANOV        # riemann_solver
    limiter: int = MC             # slope_limiter
    slope_limiting: bool = True   # useSlopeLimiting
    mood: bool = True             # fallback_2_MOOD
    precision: int = FP64

    @property
    def cells(self) -> int:
        return self.nx * self.ny

    def replace(self, **kw) -> "SolverConfig":
        d = dict(self.__dict__)
        d.update(kw)
        return SolverConfig(**d)
