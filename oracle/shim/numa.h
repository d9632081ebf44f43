/* Stand-in for <numa.h> (libnuma is not installed in this image).  The
 * reference headers call only numa_alloc_interleaved and numa_free
 * (state_vector.hpp:105,190-192,846); both map to aligned host memory.
 * Oracle build only. */
#ifndef HISV_ORACLE_NUMA_SHIM_H_
#define HISV_ORACLE_NUMA_SHIM_H_
#include <stdlib.h>
static inline void* numa_alloc_interleaved(size_t size) {
  void* p = NULL;
  if (posix_memalign(&p, 64, size ? size : 64) != 0) return NULL;
  return p;
}
static inline void numa_free(void* p, size_t size) { (void)size; free(p); }
#endif
