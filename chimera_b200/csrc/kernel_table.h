// kernel_table.h -- the instantiated kernels each precision unit exports to the
// host runtime.
#pragma once
#include <stddef.h>

namespace chimera {

struct KernelEntry {
  const void* fn;      // __global__ function (host stub address)
  size_t smem;         // dynamic shared memory bytes
  int tx, ty, nt;      // tile shape and block size
  int box_w = 0, box_h = 0;   // TMA box of the stage input (elements), 0 = plain loads
};

struct KernelSet {
  KernelEntry stage[3][3];  // [riemann-1][stage-1]
  KernelEntry cfl;
  int elem_bytes;           // storage element size
};

// Tile-shape variants per precision (for the autotuner).
int fp64_variant_count();
void fp64_kernels(int variant, KernelSet* out);
void fp64_mixed_pair_kernels(KernelSet* out);
void fp32_mixed_pair_kernels(KernelSet* out);
void fp32m_mixed_pair_kernels(KernelSet* out);
int fp32_variant_count();
void fp32_kernels(int variant, KernelSet* out);
int fp32m_variant_count();
void fp32m_kernels(int variant, KernelSet* out);

}  // namespace chimera
