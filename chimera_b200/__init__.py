"""chimera_b200: B200-native (sm_100a) per-step hot path of the CHIMERA 2-D
ideal-MHD solver -- MUSCL + MC/Van Leer + MOOD reconstruction, Rusanov/HLLE/HLLD
fluxes, constrained transport, SSP-RK3 stage combine with floors, CFL dt and
the div B monitor -- behind a C-ABI (``include/chimera_gpu.h``)."""
from .config import (BC_FIXED, BC_INFLOW, BC_OUTFLOW, BC_PERIODIC, FP32_BULK, FP32_MIXED, FP64, HLLD,
                     HLLE, MC, RUSANOV, VAN_LEER, SolverConfig)

__all__ = ["SolverConfig", "RUSANOV", "HLLE", "HLLD", "VAN_LEER", "MC", "BC_PERIODIC",
           "BC_FIXED", "BC_OUTFLOW", "BC_INFLOW", "FP64", "FP32_BULK", "FP32_MIXED"]
