// kernels_fp64.cu -- the plain FP64 form.  Compiled with --fmad=false so that
// no multiply-add is contracted and every expression rounds as the reference's
// Fortran source does (bit-compatible with the -ffp-contract=off restatement).
#include "kernel_table.h"
#include "stage_kernel.cuh"

namespace chimera {

namespace {
template <int TX, int TY, int NT, int MINB, bool KEEP_IN = false, bool TMA = false, bool MIXBC = false>
void fill(KernelSet* ks) {
  using G = TileGeom<TX, TY>;
  const int bw = TMA ? TmaBox64<TX, TY>::BW : 0, bh = TMA ? TmaBox64<TX, TY>::BH : 0;
  const size_t smem = G::template smem_bytes<double, KEEP_IN>();
#define CHIMERA_ENTRY(S, K) \
  ks->stage[S - 1][K - 1] = KernelEntry{                                                                  \
      (const void*)&stage_kernel<double, S, K, TX, TY, NT, MINB, KEEP_IN, TMA, UNIT_FP64, MIXBC>,          \
                                        smem, TX, TY, NT, bw, bh}
  CHIMERA_ENTRY(1, 1); CHIMERA_ENTRY(1, 2); CHIMERA_ENTRY(1, 3);
  CHIMERA_ENTRY(2, 1); CHIMERA_ENTRY(2, 2); CHIMERA_ENTRY(2, 3);
  CHIMERA_ENTRY(3, 1); CHIMERA_ENTRY(3, 2); CHIMERA_ENTRY(3, 3);
#undef CHIMERA_ENTRY
  ks->cfl = KernelEntry{(const void*)&cfl_kernel<double, TX, TY, NT, UNIT_FP64>, 0, TX, TY, NT};
  ks->elem_bytes = 8;
}
}  // namespace

// Tile shapes and occupancy targets the autotuner chooses from; the default
// (variant 0) loads the stage input of interior tiles by TMA.
int fp64_variant_count() { return 7; }

void fp64_kernels(int variant, KernelSet* out) {
  switch (variant) {
    case 1: fill<32, 16, 256, 2>(out); break;
    case 2: fill<32, 8, 128, 4>(out); break;
    case 3: fill<64, 8, 256, 2>(out); break;
    case 4: fill<16, 16, 128, 4>(out); break;
    case 5: fill<32, 16, 256, 2, true>(out); break;   // phase 3b reads the stage input from shared memory
    case 6: fill<32, 16, 256, 1>(out); break;
    default: fill<32, 16, 256, 2, false, true>(out); break;   // phase 1 from TMA boxes (interior tiles)
  }
}

// The one tile for grids with a periodic side facing a non-periodic one.
void fp64_mixed_pair_kernels(KernelSet* out) { fill<32, 16, 256, 2, false, false, true>(out); }

}  // namespace chimera
