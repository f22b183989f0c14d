// extern "C" entry points declared in include/symprop.h.  Each converts
// C++ exceptions into status codes and keeps the last message per thread.
#include <cstdio>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <mutex>

#include "dense.cuh"
#include "gram_tc.cuh"
#include "tensor.cuh"

namespace spb {
static thread_local std::string g_last_error;
void set_last_error(const std::string &msg) { g_last_error = msg; }


}  // namespace spb

using namespace spb;

namespace {
void require(bool ok, const char *what) {
  if (!ok) fail(SYMPROP_ERR_INVALID, "%s", what);
}
void set_current_device(const TensorState &s) { SPB_CUDA(cudaSetDevice(s.device)); }
}  // namespace

extern "C" {

const char *symprop_status_string(int status) {
  switch (status) {
    case SYMPROP_OK: return "ok";
    case SYMPROP_ERR_INVALID: return "invalid argument";
    case SYMPROP_ERR_ORDER: return "unsupported order";
    case SYMPROP_ERR_OOM: return "out of memory";
    case SYMPROP_ERR_CUDA: return "CUDA error";
    case SYMPROP_ERR_NOCONV: return "solver did not converge";
    case SYMPROP_ERR_TIMEOUT: return "device wait timed out";
    case SYMPROP_ERR_SIZE: return "size not supported";
    case SYMPROP_ERR_NODEVICE: return "no CUDA device";
    default: return "unknown status";
  }
}

const char *symprop_last_error(void) { return g_last_error.c_str(); }

int symprop_device_count(int *count) {
  return guard([&] {
    require(count, "count is null");
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) {
      cudaGetLastError();
      n = 0;
    }
    *count = n;
  });
}

int symprop_set_device(int device) {
  return guard([&] { SPB_CUDA(cudaSetDevice(device)); });
}

int symprop_trim_memory(void) {
  return guard([&] {
    SPB_CUDA(cudaDeviceSynchronize());
    SPB_CUDA(cudaMemPoolTrimTo(device_pool(), 0));
  });
}

int symprop_tensor_create(uint32_t order, uint32_t dim, const uint32_t *inds, const double *vals,
                          uint64_t nnz, symprop_tensor **out) {
  return guard([&] {
    require(out != nullptr, "out is null");
    *out = nullptr;
    require(nnz == 0 || (inds && vals), "inds/vals are null");
    require(dim > 0, "dim must be positive");
    if (order < 2 || order > 8) fail(SYMPROP_ERR_ORDER, "order %u not supported (2..8)", order);
    if (nnz * (uint64_t)order >= (1ull << 32))
      fail(SYMPROP_ERR_SIZE, "nnz*order must be below 2^32");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
      cudaGetLastError();
      fail(SYMPROP_ERR_NODEVICE, "no CUDA device visible");
    }
    auto t = std::make_unique<symprop_tensor>();
    SPB_CUDA(cudaGetDevice(&t->s.device));
    t->s.order = order;
    t->s.dim = dim;
    t->s.nnz = nnz;
    tensor_build(t->s, inds, vals);
    *out = t.release();
  });
}

int symprop_tensor_destroy(symprop_tensor *t) {
  return guard([&] {
    if (!t) return;
    cudaSetDevice(t->s.device);
    delete t;
  });
}

int symprop_tensor_order(const symprop_tensor *t, uint32_t *v) {
  return guard([&] { require(t && v, "null argument"); *v = t->s.order; });
}
int symprop_tensor_dim(const symprop_tensor *t, uint32_t *v) {
  return guard([&] { require(t && v, "null argument"); *v = t->s.dim; });
}
int symprop_tensor_nnz(const symprop_tensor *t, uint64_t *v) {
  return guard([&] { require(t && v, "null argument"); *v = t->s.nnz; });
}
int symprop_tensor_norm(const symprop_tensor *t, double *v) {
  return guard([&] { require(t && v, "null argument"); *v = t->s.norm; });
}
int symprop_tensor_owner_count(const symprop_tensor *t, uint64_t *v) {
  return guard([&] { require(t && v, "null argument"); *v = t->s.nown; });
}

int symprop_tree_build(symprop_tensor *t) {
  return guard([&] {
    require(t, "null tensor");
    set_current_device(t->s);
    tree_build(t->s);
  });
}

int symprop_tree_level_size(const symprop_tensor *t, uint32_t level, uint64_t *size) {
  return guard([&] {
    require(t && size, "null argument");
    require(t->s.tree != nullptr, "tree not built (call symprop_tree_build)");
    require(level < t->s.tree->depth, "level out of range");
    *size = t->s.tree->size[level];
  });
}

int symprop_tree_owner_count(const symprop_tensor *t, uint64_t *owners) {
  return guard([&] {
    require(t && owners, "null argument");
    require(t->s.tree != nullptr, "tree not built (call symprop_tree_build)");
    *owners = t->s.tree->nown;
  });
}

int symprop_tree_copy_level(const symprop_tensor *t, uint32_t level, uint32_t *level_idx,
                            uint64_t *level_ptr, uint64_t *dep_list) {
  return guard([&] {
    require(t, "null tensor");
    require(t->s.tree != nullptr, "tree not built (call symprop_tree_build)");
    const TreeLevels &tr = *t->s.tree;
    require(level < tr.depth, "level out of range");
    set_current_device(t->s);
    const uint64_t n = tr.size[level];
    if (level_idx && n)
      SPB_CUDA(cudaMemcpy(level_idx, tr.level_idx[level].p, n * 4, cudaMemcpyDeviceToHost));
    if (level_ptr)
      SPB_CUDA(cudaMemcpy(level_ptr, tr.level_ptr[level].p, (n + 1) * 8, cudaMemcpyDeviceToHost));
    if (dep_list && level >= 1 && n)
      SPB_CUDA(cudaMemcpy(dep_list, tr.dep_list[level].p, n * (level + 1) * 8,
                          cudaMemcpyDeviceToHost));
  });
}

int symprop_tree_copy_owners(const symprop_tensor *t, uint64_t *rem, double *val) {
  return guard([&] {
    require(t, "null tensor");
    require(t->s.tree != nullptr, "tree not built (call symprop_tree_build)");
    set_current_device(t->s);
    const TreeLevels &tr = *t->s.tree;
    if (rem && tr.nown)
      SPB_CUDA(cudaMemcpy(rem, tr.own_rem.p, tr.nown * 8, cudaMemcpyDeviceToHost));
    if (val && tr.nown)
      SPB_CUDA(cudaMemcpy(val, tr.own_val.p, tr.nown * 8, cudaMemcpyDeviceToHost));
  });
}

int symprop_s3ttmc_device(const symprop_tensor *t, const void *dU, uint32_t R, int packed,
                          void *dY, int precision, void *stream) {
  return guard([&] {
    require(t && dU && dY, "null argument");
    set_current_device(t->s);
    s3ttmc_run(const_cast<TensorState &>(t->s), dU, R, packed != 0, dY, precision,
               (cudaStream_t)stream);
  });
}

int symprop_s3ttmc(const symprop_tensor *t, const void *U, uint32_t R, int packed, void *Y,
                   int precision) {
  return guard([&] {
    require(t && U && Y, "null argument");
    require(R > 0, "R must be positive");
    require(precision == SYMPROP_FP64 || precision == SYMPROP_FP32, "unknown precision");
    TensorState &s = const_cast<TensorState &>(t->s);
    set_current_device(s);
    s3ttmc_host(s, U, R, packed != 0, Y, precision);
  });
}

int symprop_s3ttmc_schedule(int schedule) {
  return guard([&] {
    require(schedule >= 0 && schedule <= 4, "schedule must be 0, 1, 2, 3 or 4");
    set_s3ttmc_schedule(schedule);
  });
}

int symprop_s3ttmc_launches(const symprop_tensor *t, uint32_t R, int packed, uint32_t *launches) {
  return guard([&] {
    require(t && launches, "null argument");
    *launches = s3ttmc_launch_count(t->s, R, packed != 0);
  });
}

namespace {
// *d_err of a tensor-core product, read after the stream drains
void check_tc_err(cudaStream_t st, const int *d_err) {
  int h = 0;
  SPB_CUDA(cudaMemcpyAsync(&h, d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
  SPB_CUDA(cudaStreamSynchronize(st));
  if (h) fail(SYMPROP_ERR_TIMEOUT, "tensor-core product: a bounded wait expired");
}
}  // namespace

int symprop_symsyrk_device(const float *dA, const float *dscale, double *dC, uint64_t ncoeff, uint64_t I1,
                           void *stream) {
  return guard([&] {
    require(dA && dscale && dC, "null argument");
    require(ncoeff > 0 && I1 > 0 && ncoeff < (1ull << 31) && I1 < (1ull << 31), "bad sizes");
    cudaStream_t st = (cudaStream_t)stream;
    DBuf<char> ws(gram::split_bytes((int)I1, (int)ncoeff)), scr(gram::gram_rows_scratch_bytes((int)I1, (int)ncoeff));
    DBuf<int> err(1);
    SPB_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int), st));
    const gram::Split z = gram::split_view(ws.p, (int)I1, (int)ncoeff);
    gram::split(st, dA, dscale, z);
    gram::gram_rows(st, z, dC, scr.p, err.p);
    check_tc_err(st, err.p);
  });
}

int symprop_symgemm_device(const float *dA, const double *dB, const double *dscale, double *dC,
                           uint64_t ncoeff, uint64_t I1, uint64_t I2, void *stream) {
  return guard([&] {
    require(dA && dB && dscale && dC, "null argument");
    require(ncoeff > 0 && I1 > 0 && I2 > 0 && ncoeff < (1ull << 31) && I1 < (1ull << 31) && I2 < (1ull << 20),
            "bad sizes");
    cudaStream_t st = (cudaStream_t)stream;
    DBuf<char> ws(gram::split_bytes((int)I1, (int)ncoeff)), scr(gram::times_scratch_bytes((int)I1, (int)ncoeff));
    DBuf<float> sc((size_t)ncoeff);
    DBuf<int> err(1);
    SPB_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int), st));
    dense::convert<double, float>(st, dscale, sc.p, (size_t)ncoeff);
    const gram::Split z = gram::split_view(ws.p, (int)I1, (int)ncoeff);
    gram::split(st, dA, sc.p, z);
    for (uint64_t q0 = 0; q0 < I2; q0 += gram::kPanelRows)
      gram::times(st, z, dB + q0 * ncoeff, (int)std::min<uint64_t>(gram::kPanelRows, I2 - q0), (size_t)ncoeff, 1,
                  dscale, dC + q0, (size_t)I2, scr.p, err.p);
    check_tc_err(st, err.p);
  });
}

int symprop_gram_device(const void *dY, uint64_t n, uint32_t m, const void *dscale, double *dG,
                        int precision, void *stream) {
  return guard([&] {
    require(dY && dscale && dG, "null argument");
    require(n > 0 && m > 0 && n < (1ull << 31), "bad sizes");
    cudaStream_t st = (cudaStream_t)stream;
    if (precision == SYMPROP_FP64) {
      const double *Y = (const double *)dY, *sd = (const double *)dscale;
      dense::gemm<double>(st, (int)m, (int)m, (int)n, 1.0, Y, (int)m, true, Y, (int)m, false, 0.0, dG,
                          (int)m, nullptr, true);
      dense::scale_sym(st, dG, (int)m, sd);
    } else if (precision == SYMPROP_FP32) {
      DBuf<char> ws(gram::workspace_bytes((int)n, (int)m));
      DBuf<int> err(1);
      SPB_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int), st));
      gram::gram_split_bf16(st, (const float *)dY, (int)n, (int)m, (const float *)dscale, dG, ws.p,
                            err.p);
      int h = 0;
      SPB_CUDA(cudaMemcpyAsync(&h, err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
      SPB_CUDA(cudaStreamSynchronize(st));
      if (h) fail(SYMPROP_ERR_TIMEOUT, "tensor-core Gram: a bounded wait expired");
    } else {
      fail(SYMPROP_ERR_INVALID, "unknown precision");
    }
    SPB_CUDA(cudaStreamSynchronize(st));
  });
}

uint64_t symprop_symtens_size(uint32_t dim, uint32_t order) { return symsize(dim, order); }

int symprop_symtens_coeff(uint32_t dim, uint32_t order, double *coeff) {
  return guard([&] {
    require(coeff, "null argument");
    for_each_sorted(dim, (int)order, [&](const std::vector<uint32_t> &q, uint64_t lin) {
      uint64_t denom = 1, run = 1;
      for (size_t j = 1; j <= q.size(); ++j) {
        if (j < q.size() && q[j] == q[j - 1]) {
          ++run;
        } else {
          denom *= factorial_u64((int)run);
          run = 1;
        }
      }
      coeff[lin] = (double)(factorial_u64((int)order) / denom);
    });
  });
}

int symprop_unpack_rows_device(const double *dpacked, uint64_t rows, uint32_t dim, uint32_t order,
                               double *dfull, void *stream) {
  return guard([&] {
    require(dpacked && dfull, "null argument");
    unpack_rows(dpacked, rows, dim, order, dfull, SYMPROP_FP64, (cudaStream_t)stream);
  });
}

int symprop_write_decomp(const char *path, const double *core, const double *factor, uint32_t dim,
                         uint32_t rank, uint32_t order, int append) {
  return guard([&] {
    require(path && core && factor, "null argument");
    std::string p = path;
    if (p.empty()) return;
    if (p == "stdout") p = "/dev/stdout";
    if (p == "stderr") p = "/dev/stderr";
    std::ofstream os(p, append ? std::ios::app : std::ios::out);
    if (!os) fail(SYMPROP_ERR_INVALID, "cannot open %s", path);
    // SymTuckerDecomp::print (src/tucker.cpp:47-61), including its row
    // stride of `rank` into the rank x rank^(order-1) core.
    uint64_t csize = 1;
    for (uint32_t j = 0; j < order; ++j) csize *= rank;
    os << "Mode-1 matricized C:\n";
    for (uint64_t i = 0; i < rank; ++i) {
      for (uint64_t j = 0; j < csize / rank; ++j) os << core[i * rank + j] << ",";
      os << "\n";
    }
    os << "Factor U:\n";
    for (uint64_t i = 0; i < dim; ++i) {
      for (uint64_t j = 0; j < rank; ++j) os << factor[i * rank + j] << ",";
      os << "\n";
    }
  });
}

}  // extern "C"
