// Bounds checks of the checked build (-DSYMPROP_CHECK, `make checked`,
// libsymprop_b200_checked.so).  In that build SPB_BOUND(cond, site, value)
// tests cond on the device; a failed check records its site and value in
// this translation unit's flag and the access it guards is skipped, so a
// wrong index becomes a status code instead of a fault.  The launch wrappers
// read the flag after their kernels (spb_check_host) and raise
// SYMPROP_ERR_CUDA naming the site.  In the normal build SPB_BOUND is the
// constant true and every check compiles away.
#pragma once

#include "common.cuh"

namespace spb {

#ifdef SYMPROP_CHECK
// one flag per translation unit (the kernels of each .cu are a separate
// module); site 0 = no failure
static __device__ unsigned int g_check_site;
static __device__ unsigned long long g_check_value;

__device__ __forceinline__ bool spb_check_fail(unsigned int site, unsigned long long value) {
  if (atomicCAS(&g_check_site, 0u, site) == 0u) g_check_value = value;
  return false;
}
#define SPB_BOUND(cond, site, value) ((cond) ? true : ::spb::spb_check_fail((site), (unsigned long long)(value)))

// Waits for `st`, then fails with the first recorded site (and clears it).
static inline void spb_check_host(cudaStream_t st, const char *what) {
  SPB_CUDA(cudaStreamSynchronize(st));
  unsigned int site = 0;
  unsigned long long value = 0;
  SPB_CUDA(cudaMemcpyFromSymbol(&site, g_check_site, sizeof(site)));
  if (!site) return;
  SPB_CUDA(cudaMemcpyFromSymbol(&value, g_check_value, sizeof(value)));
  const unsigned int zero = 0;
  SPB_CUDA(cudaMemcpyToSymbol(g_check_site, &zero, sizeof(zero)));
  fail(SYMPROP_ERR_CUDA, "%s: device bounds check %u failed (value %llu)", what, site, value);
}
#else
#define SPB_BOUND(cond, site, value) true
static inline void spb_check_host(cudaStream_t, const char *) {}
#endif

}  // namespace spb
