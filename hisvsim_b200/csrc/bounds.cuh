// Index checks of the bounds-checked build (compiled with -DHS_BOUNDS into
// libhisv_bounds.so; the stand-in for a memory checker): every global and
// shared-memory access of the K1, K2, K4 and K6 kernels is guarded by
// HS_IN_BOUNDS(condition, kernel bit).  A failed check sets the kernel's bit
// in a device flag of its translation unit and skips the access;
// hs_bounds_status reads the flags.  In the normal build the checks are the
// constant true and compile to nothing.
#pragma once

#include <cuda_runtime.h>

namespace hisv {

constexpr unsigned kBoundsK1 = 1u, kBoundsK2 = 2u, kBoundsK4 = 4u, kBoundsK6 = 8u;

#ifdef HS_BOUNDS
namespace {
__device__ unsigned int g_bounds_flag;  // one per translation unit
}  // namespace
#define HS_IN_BOUNDS(cond, bit) ((cond) || (atomicOr(&g_bounds_flag, (bit)), false))
// host: read (and optionally clear) this translation unit's flag
#define HS_BOUNDS_TAKE(fn)                                                    \
  unsigned fn(int reset) {                                                    \
    unsigned v = 0;                                                           \
    cudaMemcpyFromSymbol(&v, g_bounds_flag, sizeof(v));                       \
    if (reset) {                                                              \
      const unsigned z = 0;                                                   \
      cudaMemcpyToSymbol(g_bounds_flag, &z, sizeof(z));                       \
    }                                                                         \
    return v;                                                                 \
  }
#else
#define HS_IN_BOUNDS(cond, bit) true
#endif

// the flags of the four kernel files (bounds-checked build only)
unsigned bounds_take_part(int reset);
unsigned bounds_take_misc(int reset);
unsigned bounds_take_fused(int reset);
unsigned bounds_take_batch(int reset);

}  // namespace hisv
