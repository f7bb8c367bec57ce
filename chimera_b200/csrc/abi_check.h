// abi_check.h -- checks of caller pointers at the C-ABI, made before any
// device call.  The kernels behind chimera_rk3_step_noalloc, chimera_op_* and
// the adjoint steps read and write the caller's arrays as doubles, so a null or
// misaligned address is refused with CHIMERA_ERR_BAD_ARG instead of reaching a
// launch (where it would fault).
#pragma once
#include <stdint.h>

#include <initializer_list>

namespace chimera {

inline bool double_ok(const void* p) { return p && (reinterpret_cast<uintptr_t>(p) & 7u) == 0; }

inline bool doubles_ok(std::initializer_list<const void*> ptrs) {
  for (const void* p : ptrs)
    if (!double_ok(p)) return false;
  return true;
}

}  // namespace chimera
