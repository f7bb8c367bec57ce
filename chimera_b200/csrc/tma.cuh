// tma.cuh -- tensor-memory-accelerator (TMA) box copies into shared memory,
// completed on a shared-memory mbarrier.  Plain tiled 2-D loads of this GPU's
// own memory: no cluster multicast anywhere.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace chimera {

constexpr int TMAP_BYTES = 128;   // sizeof(CUtensorMap)

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Order this thread's earlier generic-proxy accesses of shared memory (made
// visible to it by a barrier) before the async-proxy writes it issues next.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// One arrival that also announces `bytes` of transaction to come.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

// The box of the 2-D tensor map `tmap` (in global memory) whose first element
// is at (x, y) -> shared memory at dst; completes `bar`'s transaction count.
// x times the element size must be a multiple of 16 bytes.
__device__ __forceinline__ void tma_load_2d(void* dst, const void* tmap, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(tmap)), "r"(x), "r"(y), "r"(smem_addr(bar))
      : "memory");
}

// Wait for the phase with parity `parity` of `bar` to complete, giving up
// after max_iter polls; returns whether it completed.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, unsigned max_iter) {
  for (unsigned it = 0; it < max_iter; ++it) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

}  // namespace chimera
