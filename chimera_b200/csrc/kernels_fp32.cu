// kernels_fp32.cu -- the FP32-bulk form (stage_kernel_f32).  Compiled with
// -use_fast_math: FP32 division and square root are the fast (about 1 ulp)
// forms; the FP64 parts (pressure recovery, dt reduction, sums) are unaffected.
#include "kernel_table.h"
#include "stage_kernel_fp32.cuh"

namespace chimera {

namespace {
// Storage type ST: float (FP32-bulk) or double (FP32 arithmetic on FP64
// storage, whose CFL kernel has the FP64 epilogue's arithmetic; compiled in this
// unit, its own instantiation).
template <int TX, int TY, int NT, int MINB, bool SB = true, bool TMA = false, typename ST = float,
          bool MIXBC = false>
void fill(KernelSet* ks) {
  using G = TileGeom32<TX, TY, SB>;
  const size_t smem = G::smem_bytes();
  const int bw = TMA ? G::BW : 0, bh = TMA ? G::BH : 0;
#define CHIMERA_ENTRY(S, K)                                                                            \
  ks->stage[S - 1][K - 1] =                                                                           \
      KernelEntry{(const void*)&stage_kernel_f32<S, K, TX, TY, NT, MINB, SB, TMA, ST, MIXBC>, smem, TX, TY, NT, \
                  bw, bh}
  CHIMERA_ENTRY(1, 1); CHIMERA_ENTRY(1, 2); CHIMERA_ENTRY(1, 3);
  CHIMERA_ENTRY(2, 1); CHIMERA_ENTRY(2, 2); CHIMERA_ENTRY(2, 3);
  CHIMERA_ENTRY(3, 1); CHIMERA_ENTRY(3, 2); CHIMERA_ENTRY(3, 3);
#undef CHIMERA_ENTRY
  ks->cfl = KernelEntry{(const void*)&cfl_kernel<ST, TX, TY, NT, UNIT_FP32>, 0, TX, TY, NT};
  ks->elem_bytes = int(sizeof(ST));
}
}  // namespace

// Tile shapes and occupancy targets the autotuner chooses from.
int fp32_variant_count() { return 11; }

void fp32_kernels(int variant, KernelSet* out) {
  switch (variant) {
    case 1: fill<32, 8, 128, 3>(out); break;
    case 2: fill<64, 8, 256, 2>(out); break;
    case 3: fill<16, 16, 128, 4>(out); break;
    case 4: fill<32, 16, 512, 1>(out); break;
    case 5: fill<32, 16, 256, 3, false>(out); break;
    case 6: fill<16, 16, 128, 6, false>(out); break;
    case 7: fill<32, 8, 128, 5, false>(out); break;
    case 8: fill<64, 8, 256, 2, false>(out); break;
    case 9: fill<32, 16, 256, 3, false, true>(out); break;
    case 10: fill<16, 16, 128, 6, false, true>(out); break;
    default: fill<32, 16, 256, 2>(out); break;
  }
}

// The FP32-arithmetic form on FP64 storage: the FP32-bulk tiles without TMA.
int fp32m_variant_count() { return 4; }

void fp32m_kernels(int variant, KernelSet* out) {
  switch (variant) {
    case 1: fill<32, 16, 256, 3, false, false, double>(out); break;
    case 2: fill<32, 8, 128, 5, false, false, double>(out); break;
    case 3: fill<16, 16, 128, 6, false, false, double>(out); break;
    default: fill<32, 16, 256, 2, true, false, double>(out); break;
  }
}

// The one tile of each form for grids with a periodic side facing a non-periodic one.
void fp32_mixed_pair_kernels(KernelSet* out) { fill<32, 16, 256, 2, true, false, float, true>(out); }
void fp32m_mixed_pair_kernels(KernelSet* out) { fill<32, 16, 256, 2, true, false, double, true>(out); }

}  // namespace chimera
