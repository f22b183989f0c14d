// Shared host/device utilities of the symprop_b200 library: error plumbing
// (C-ABI status codes + per-thread message), device buffers, and the packed
// symmetric-index arithmetic of the reference
// (include/detail/dense/symtensor_base.hpp:12-30, 42-76).
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "symprop.h"

namespace spb {

// ----------------------------------------------------------------- errors

struct Error : std::exception {
  int code;
  std::string msg;
  Error(int c, std::string m) : code(c), msg(std::move(m)) {}
  const char *what() const noexcept override { return msg.c_str(); }
};

void set_last_error(const std::string &msg);

[[noreturn]] inline void fail(int code, const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  throw Error(code, buf);
}

inline void cuda_check(cudaError_t e, const char *what, const char *file, int line) {
  if (e != cudaSuccess) {
    // reset the runtime's last-error slot: a refused allocation (or another
    // non-sticky error) would otherwise resurface at the next launch check
    cudaGetLastError();
    int code = (e == cudaErrorMemoryAllocation) ? SYMPROP_ERR_OOM
               : (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
                   ? SYMPROP_ERR_NODEVICE
                   : SYMPROP_ERR_CUDA;
    fail(code, "%s failed: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
  }
}
#define SPB_CUDA(x) ::spb::cuda_check((x), #x, __FILE__, __LINE__)
#define SPB_LAUNCH_CHECK() ::spb::cuda_check(cudaGetLastError(), "kernel launch", __FILE__, __LINE__)

// Runs `body` and converts exceptions into a status code (C-ABI boundary).
template <class F> int guard(F &&body) {
  try {
    body();
    return SYMPROP_OK;
  } catch (const Error &e) {
    set_last_error(e.msg);
    return e.code;
  } catch (const std::bad_alloc &) {
    set_last_error("host allocation failed");
    return SYMPROP_ERR_OOM;
  } catch (const std::exception &e) {
    set_last_error(e.what());
    return SYMPROP_ERR_INVALID;
  }
}

// ------------------------------------------------------------ NVTX ranges
// Named host phases for nsys / ncu --nvtx (the GPU counterpart of the
// reference's FunctionTimer scopes, src/utils/function_timer.cpp); the calls
// do nothing unless a profiling tool is attached.
struct NvtxRange {
  explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange &) = delete;
  NvtxRange &operator=(const NvtxRange &) = delete;
};

// ---------------------------------------------------------- device buffer

template <class T> struct DBuf {
  T *p = nullptr;
  size_t n = 0;
  DBuf() = default;
  explicit DBuf(size_t count) { alloc(count); }
  DBuf(const DBuf &) = delete;
  DBuf &operator=(const DBuf &) = delete;
  DBuf(DBuf &&o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
  DBuf &operator=(DBuf &&o) noexcept {
    if (this != &o) { release(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
    return *this;
  }
  ~DBuf() { release(); }
  void alloc(size_t count) {
    release();
    if (count == 0) return;
    SPB_CUDA(cudaMalloc(&p, count * sizeof(T)));
    n = count;
  }
  // grows (never shrinks); contents are not preserved
  void ensure(size_t count) {
    if (count > n) alloc(count);
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  size_t bytes() const { return n * sizeof(T); }
};

// The library's stream-ordered memory pool of the current device (dense.cu).
cudaMemPool_t device_pool();

// ------------------------------------------------------- packed indexing

inline uint64_t binom(uint64_t n, uint64_t k) {
  if (k > n) return 0;
  if (2 * k > n) k = n - k;
  if (k == 0) return 1;
  uint64_t r = n;
  for (uint64_t i = 2; i <= k; ++i) {
    r *= (n - i + 1);
    r /= i;
  }
  return r;
}
// number of sorted order-`order` multi-indices over [0, dim)
inline uint64_t symsize(uint64_t dim, uint64_t order) { return binom(order + dim - 1, order); }

__host__ __device__ inline uint64_t factorial_u64(int k) {
  uint64_t f = 1;
  for (int i = 2; i <= k; ++i) f *= (uint64_t)i;
  return f;
}

// Host enumeration of sorted multi-indices of length `order` over [0,dim) in
// the reference's lexicographic packed order.  Calls f(idx, linear).
template <class F> void for_each_sorted(uint32_t dim, int order, F &&f) {
  std::vector<uint32_t> q((size_t)order, 0);
  uint64_t lin = 0;
  if (dim == 0) return;
  if (order == 0) { f(q, lin); return; }
  while (true) {
    f(q, lin);
    ++lin;
    int j = order - 1;
    while (j >= 0 && q[(size_t)j] + 1 >= dim) --j;
    if (j < 0) break;
    q[(size_t)j]++;
    for (int k = j + 1; k < order; ++k) q[(size_t)k] = q[(size_t)j];
  }
}

inline int bits_for(uint64_t v) {  // bits to hold values in [0, v]
  int b = 1;
  while ((v >> b) != 0) ++b;
  return b;
}

}  // namespace spb
