// kernels_fp32.cu -- the FP32-bulk form: FP32 storage and bulk reconstruction /
// flux arithmetic (FMA contraction allowed); the CFL dt, div B and the
// conserved totals are reduced in FP64.
#include "kernel_table.h"
#include "stage_kernel.cuh"

namespace chimera {

namespace {
template <int TX, int TY, int NT, int MINB>
void fill(KernelSet* ks) {
  using G = TileGeom<TX, TY>;
  const size_t smem = G::template smem_bytes<float>();
#define CHIMERA_ENTRY(S, K) \
  ks->stage[S - 1][K - 1] = KernelEntry{(const void*)&stage_kernel<float, S, K, TX, TY, NT, MINB>, smem, TX, TY, NT}
  CHIMERA_ENTRY(1, 1); CHIMERA_ENTRY(1, 2); CHIMERA_ENTRY(1, 3);
  CHIMERA_ENTRY(2, 1); CHIMERA_ENTRY(2, 2); CHIMERA_ENTRY(2, 3);
  CHIMERA_ENTRY(3, 1); CHIMERA_ENTRY(3, 2); CHIMERA_ENTRY(3, 3);
#undef CHIMERA_ENTRY
  ks->cfl = KernelEntry{(const void*)&cfl_kernel<float, TX, TY, NT>, 0, TX, TY, NT};
  ks->elem_bytes = 4;
}
}  // namespace

// Tile shapes and occupancy targets the autotuner chooses from.
int fp32_variant_count() { return 5; }

void fp32_kernels(int variant, KernelSet* out) {
  switch (variant) {
    case 1: fill<32, 16, 256, 2>(out); break;
    case 2: fill<32, 8, 128, 4>(out); break;
    case 3: fill<64, 8, 256, 2>(out); break;
    case 4: fill<16, 16, 128, 4>(out); break;
    default: fill<32, 16, 256, 1>(out); break;
  }
}

}  // namespace chimera
