// Tucker drivers on the GPU: HOOI, HOQRI and AltHOOI with the reference's
// control flow, stopping rule and printed lines.
//
//   TuckerHOOI    src/sparse/spsymtensor.cpp:201-252
//   TuckerHOQRI   src/sparse/spsymtensor.cpp:254-299
//   TuckerAltHOOI src/sparse/spsymtensor.cpp:301-337
//   regularize    src/sparse/spsymtensor.cpp:168-199
//   random init   src/tucker.cpp:25-36 (std::mt19937(seed) +
//                 std::normal_distribution<double>(0,1), row-major dim x rank)
//   hosvd_init    src/sparse/spsymtensor.cpp:339-383
//   error         src/tucker.cpp:40-45: sqrt(||X||^2 - ||C||^2) / ||X||
//
// HOOI's leftsvd of the unpacked n x R^(N-1) Y is replaced by the packed
// Gram: Y_unp Y_unp^T = Y D Y^T with D the permutation counts of the packed
// columns (every packed column appears D_q times in the unpacked Y), so the
// leading left singular subspace is the top-r eigenspace of Y D Y^T
// (n <= m) or U = orth(Y D^1/2 V) with V the top-r eigenvectors of
// D^1/2 Y^T Y D^1/2 (n > m).  ||C||^2 of the unpacked core is the
// D-weighted norm of the packed core U^T Y.  Every later step is invariant
// under U -> U Q for orthogonal Q, so the error trajectory does not depend on
// which orthonormal basis LAPACK or this code returns; the printed "relative
// residual" compares cores in those bases and is basis-dependent.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <future>
#include <iomanip>
#include <iostream>
#include <random>
#include <vector>

#include "dense.cuh"
#include "gram_tc.cuh"
#include "tensor.cuh"

namespace spb {
namespace {

__global__ void scale_sym_kernel(double *G, int m, const double *sd) {
  size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (size_t)m * m) return;
  int i = (int)(idx / m), j = (int)(idx % m);
  G[idx] *= sd[i] * sd[j];
}

// A += mult(C) w_C w_C^T over the leaves C of the tree (hoevd init):
// A = X_(1) X_(1)^T (src/sparse/spsymtensor.cpp:385-439).
__global__ void hoevd_syrk_kernel(const uint64_t *own_ptr, const uint64_t *rem, const double *val,
                                  const double *leaf_mult, uint64_t nleaf, int n, double *A) {
  uint64_t leaf = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (leaf >= nleaf) return;
  uint64_t b = own_ptr[leaf], e = own_ptr[leaf + 1];
  double mult = leaf_mult[leaf];
  for (uint64_t i = b; i < e; ++i) {
    if (i > b && rem[i] == rem[i - 1]) continue;  // repeated ids give duplicate owners
    for (uint64_t j = i; j < e; ++j) {
      if (j > i && rem[j] == rem[j - 1]) continue;
      uint64_t p = rem[i] - 1, q = rem[j] - 1;
      double v = mult * val[i] * val[j];
      atomicAdd(&A[p * n + q], v);
      if (p != q) atomicAdd(&A[q * n + p], v);
    }
  }
}

struct Timer {
  cudaEvent_t a, b;
  cudaStream_t st;
  explicit Timer(cudaStream_t s) : st(s) {
    SPB_CUDA(cudaEventCreate(&a));
    SPB_CUDA(cudaEventCreate(&b));
  }
  ~Timer() {
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  }
  void start() { SPB_CUDA(cudaEventRecord(a, st)); }
  double stop_ms() {
    SPB_CUDA(cudaEventRecord(b, st));
    SPB_CUDA(cudaEventSynchronize(b));
    float ms = 0;
    SPB_CUDA(cudaEventElapsedTime(&ms, a, b));
    return ms;
  }
};

void regularize(cudaStream_t st, double *U, int n, int r, double delta) {
  dense::scale_rows_clip(st, U, n, r, delta);
  dense::orthonormalize(st, U, n, r);  // leftsvd(U) -> any orthonormal basis of its span
}

// The reference prints LAPACK's failure and carries on with the result
// (src/dense/matrixops.cpp:31-33, 86-89); the eigensolver here does the same.
void warn_noconv(int alg) {
  std::printf(alg == SYMPROP_ALTHOOI ? "Eigendecomposition failed to converge.\n"
                                     : "SVD failed to converge.\n");
  std::fflush(stdout);
}

}  // namespace

void hoevd_factor(TensorState &t, cudaStream_t st, int r, double *U, bool print_matrix);
int hoevd_matrix_free(TensorState &t, cudaStream_t st, int r, double *U);
// largest n whose n x n hoevd matrix is formed (and printed under verbose
// output, as the reference prints it); above it the matrix-free path
constexpr int kHoevdDenseMax = 8192;

int run_tucker(TensorState &t, const symprop_config &c, int alg, symprop_result &res) {
  NvtxRange nv(alg == SYMPROP_HOOI ? "TuckerHOOI" : alg == SYMPROP_HOQRI ? "TuckerHOQRI" : "TuckerAltHOOI");
  const int n = (int)t.dim, N = (int)t.order, r = (int)c.rank;
  if (r < 1) fail(SYMPROP_ERR_INVALID, "rank must be positive");
  if (r > n) fail(SYMPROP_ERR_INVALID, "rank %d exceeds dim %d", r, n);
  if (N < 3) fail(SYMPROP_ERR_ORDER, "Tucker needs order >= 3");
  if (alg < 0 || alg > 2) fail(SYMPROP_ERR_INVALID, "unknown algorithm %d", alg);
  const bool mixed = c.precision == SYMPROP_PREC_MIXED;
  const int L = N - 1;
  const uint64_t m64 = symsize(r, L);
  if (m64 > (1u << 30)) fail(SYMPROP_ERR_SIZE, "packed width too large");
  const int m = (int)m64;
  uint64_t full = 1;
  for (int j = 0; j < L; ++j) full *= (uint64_t)r;
  const double normX = t.norm;

  cudaStream_t st;
  SPB_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() { cudaStreamDestroy(s); }
  } sg{st};
  Timer tall(st), tphase(st), titer(st);
  auto wall0 = std::chrono::steady_clock::now();
  tall.start();

  // packed-column weights D (src/dense/symtensor.cpp:53-59)
  std::vector<double> hD(m), hsD(m);
  for_each_sorted((uint32_t)r, L, [&](const std::vector<uint32_t> &q, uint64_t lin) {
    uint64_t denom = 1, run = 1;
    for (size_t j = 1; j <= q.size(); ++j) {
      if (j < q.size() && q[j] == q[j - 1]) ++run;
      else { denom *= factorial_u64((int)run); run = 1; }
    }
    hD[lin] = (double)(factorial_u64(L) / denom);
    hsD[lin] = std::sqrt(hD[lin]);
  });
  DBuf<double> dD(m), dsD(m);
  SPB_CUDA(cudaMemcpy(dD.p, hD.data(), sizeof(double) * m, cudaMemcpyHostToDevice));
  SPB_CUDA(cudaMemcpy(dsD.p, hsD.data(), sizeof(double) * m, cudaMemcpyHostToDevice));

  // the reference's random factor (std::mt19937(seed), N(0, 1), row-major;
  // src/tucker.cpp:25-36), drawn on a host thread while the
  // device buffers are allocated and the S3TTMc layout is built; a user
  // factor replaces it (and needs no draw)
  const bool user_init = c.init == SYMPROP_INIT_USER;
  if (user_init && !res.init_factor) fail(SYMPROP_ERR_INVALID, "init_factor is null");
  std::vector<double> h0((size_t)n * r);
  std::future<void> rng;
  if (user_init) {
    std::copy(res.init_factor, res.init_factor + h0.size(), h0.begin());
  } else {
    rng = std::async(std::launch::async, [&h0, seed = c.seed] {
      std::normal_distribution<double> distr(0.0, 1.0);
      std::mt19937 engine{(std::mt19937::result_type)seed};
      for (double &x : h0) x = distr(engine);
    });
  }
  DBuf<double> U((size_t)n * r), Uprev((size_t)n * r);
  s3ttmc_prepare(t, (uint32_t)r, true, mixed ? SYMPROP_FP32 : SYMPROP_FP64);

  const bool gram_nn = n <= m;  // n x n form (AltHOOI's symsyrk) vs m x m Gram
  const int s = gram_nn ? n : m;
  // FP64 Y: allocated when an FP64 S3TTMc first runs (the mixed driver may
  // finish in FP64)
  DBuf<double> Y(mixed ? 0 : (size_t)n * m);
  // mixed: FP32 Y and U, the split-BF16 operand Z = Y D^1/2 ~ H + L and the
  // tensor-core products' scratch
  DBuf<float> Y32(mixed ? (size_t)n * m : 0), U32(mixed ? (size_t)n * r : 0), sD32(mixed ? m : 0);
  DBuf<char> split_ws(mixed ? gram::split_bytes(n, m) : 0);
  DBuf<char> gram_scr(mixed && alg != SYMPROP_HOQRI
                          ? (gram_nn ? gram::gram_rows_scratch_bytes(n, m) : gram::gram_cols_scratch_bytes(n, m))
                          : 0);
  DBuf<char> times_scr(mixed ? gram::times_scratch_bytes(n, m) : 0);
  const gram::Split Z = mixed ? gram::split_view(split_ws.p, n, m) : gram::Split{};
  if (mixed) dense::convert<double, float>(st, dsD.p, sD32.p, m);
  DBuf<int> gram_err(1);
  SPB_CUDA(cudaMemsetAsync(gram_err.p, 0, sizeof(int), st));
  // W (n x r) = Z P^T on the tensor cores, 16 columns of W per product
  auto tc_times = [&](const double *P, size_t sq, size_t sk, const double *colscale, double *W) {
    for (int q0 = 0; q0 < r; q0 += gram::kPanelRows)
      gram::times(st, Z, P + q0 * sq, std::min(gram::kPanelRows, r - q0), sq, sk, colscale, W + q0,
                  (size_t)r, times_scr.p, gram_err.p);
  };
  DBuf<double> S((size_t)s * s), V((size_t)s * r), Vwarm((size_t)s * r);
  DBuf<double> core((size_t)r * m), core_prev((size_t)r * m), red(2);
  SPB_CUDA(cudaMemsetAsync(core_prev.p, 0, sizeof(double) * r * m, st));
  // factor initialisation
  if (rng.valid()) rng.get();
  SPB_CUDA(cudaMemcpy(U.p, h0.data(), sizeof(double) * h0.size(), cudaMemcpyHostToDevice));
  // AltHOOI keeps the factor before hosvd_init as factor_prev (spsymtensor.cpp:306-308)
  SPB_CUDA(cudaMemcpy(Uprev.p, h0.data(), sizeof(double) * h0.size(), cudaMemcpyHostToDevice));
  if (c.init == SYMPROP_INIT_HOSVD) {
    // non-MKL reference build: prints and leaves the random factor
    // (src/sparse/matrixops.cpp:15-17)
    std::printf("Error: sparse SVD requires MKL.\n");
    std::fflush(stdout);
  } else if (c.init == SYMPROP_INIT_HOEVD) {
    hoevd_factor(t, st, r, U.p, c.verbose != 0);
  }
  bool have_warm = false;
  std::vector<double> lam(r);
  // Mixed precision: the objective and the convergence test are FP64 (the
  // core U^T Y is formed in FP64 from the FP32 Y).  The FP32 S3TTMc carries
  // a relative error of about 1e-7 (measured 1.2e-7) into ||C||^2, which
  // moves error = sqrt(1 - ||C||^2/||X||^2) by about
  //     noise = (||C||^2/||X||^2) * 1e-7 / (2 error).
  // While the tolerance is at least 4 x noise the mixed iteration stops on
  // its own test; otherwise it runs down to 4 x noise and finishes with FP64
  // iterations, so the final objective is within the tolerance of the FP64
  // fixed point's either way.
  constexpr double kMixedRel = 1e-7;
  double fp64_eig_tol = 1e-12;
  if (const char *e = std::getenv("SPB_EIG_TOL")) fp64_eig_tol = std::max(std::atof(e), 1e-15);
  bool mx = mixed;

  double prev_error = 0.0, error = 0.0, cn2 = 0.0;
  double s3_ms = 0, dense_ms = 0;
  // SPB_TRACE_TUCKER=1 prints each iteration's precision, phase times and error
  const char *tr = std::getenv("SPB_TRACE_TUCKER");
  const bool trace = tr && *tr && *tr != '0';
  double s3_prev = 0, dense_prev = 0;
  uint64_t iters = 0;
  int status = SYMPROP_OK;
  const int prec_digits = alg == SYMPROP_ALTHOOI ? 10 : 12;

  if (trace)
    std::fprintf(stderr, "tucker: setup %.1f ms (buffers, init)\n",
                 std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - wall0).count());
  for (uint64_t iter = 0; iter < c.max_iter; ++iter) {
    if (trace) titer.start();
    // eigen-residual target relative to the largest eigenvalue: the FP32 /
    // split-BF16 Gram of the mixed phase resolves about 1e-6 of it
    const double eig_tol = mx ? 1e-5 : fp64_eig_tol;
    nvtxRangePushA("regularize");
    tphase.start();
    regularize(st, U.p, n, r, c.delta);
    dense_ms += tphase.stop_ms();
    nvtxRangePop();

    tphase.start();
    if (mx) {
      dense::convert<double, float>(st, U.p, U32.p, (size_t)n * r);
      s3ttmc_run(t, U32.p, (uint32_t)r, true, Y32.p, SYMPROP_FP32, st);
    } else {
      Y.ensure((size_t)n * m);
      s3ttmc_run(t, U.p, (uint32_t)r, true, Y.p, SYMPROP_FP64, st);
    }
    s3_ms += tphase.stop_ms();
    const bool tc = mx;  // this iteration's dense products run on the tensor cores

    nvtxRangePushA("dense step");
    tphase.start();
    double rel_res = 0.0;
    if (alg == SYMPROP_HOOI || alg == SYMPROP_ALTHOOI) {
      // leading r-dimensional left singular subspace of Y D^1/2
      if (gram_nn) {
        if (mx) {
          // tensor-core split-BF16 Gram of the rows of Y D^1/2 (FP32 accumulation)
          gram::split(st, Y32.p, sD32.p, Z);
          gram::gram_rows(st, Z, S.p, gram_scr.p, gram_err.p);
        } else {
          dense::gemm<double>(st, n, n, m, 1.0, Y.p, m, false, Y.p, m, true, 0.0, S.p, n, dD.p, true);
        }
        int e = dense::top_eigs(st, S.p, n, r, V.p, lam.data(), have_warm ? Vwarm.p : nullptr,
                                eig_tol, 60);
        if (e != SYMPROP_OK) warn_noconv(alg);
        SPB_CUDA(cudaMemcpyAsync(U.p, V.p, sizeof(double) * n * r, cudaMemcpyDeviceToDevice, st));
      } else {
        if (mx) {
          // tensor-core split-BF16 Gram of the columns of Y D^1/2
          gram::split(st, Y32.p, sD32.p, Z);
          gram::gram_cols(st, Z, S.p, gram_scr.p, gram_err.p);
        } else {
          dense::gemm<double>(st, m, m, n, 1.0, Y.p, m, true, Y.p, m, false, 0.0, S.p, m, nullptr, true);
          scale_sym_kernel<<<(unsigned)(((size_t)m * m + 255) / 256), 256, 0, st>>>(S.p, m, dsD.p);
          SPB_LAUNCH_CHECK();
        }
        int e = dense::top_eigs(st, S.p, m, r, V.p, lam.data(), have_warm ? Vwarm.p : nullptr,
                                eig_tol, 60);
        if (e != SYMPROP_OK) warn_noconv(alg);
        if (mx) {
          tc_times(V.p, 1, (size_t)r, nullptr, U.p);  // U = Y D^1/2 V (P = V^T)
        } else {
          dense::gemm<double>(st, n, r, m, 1.0, Y.p, m, false, V.p, r, false, 0.0, U.p, r, dsD.p);
        }
        dense::orthonormalize(st, U.p, n, r);
      }
      SPB_CUDA(cudaMemcpyAsync(Vwarm.p, V.p, sizeof(double) * (size_t)s * r, cudaMemcpyDeviceToDevice, st));
      have_warm = true;
      // core = U^T Y (r x m packed), FP64 in both modes: the objective and
      // the convergence test read it (mixed: from the FP32 Y, widened in
      // registers)
      if (mx) dense::core_from_f32(st, U.p, Y32.p, n, m, r, core.p);
      else dense::core_from_f64(st, U.p, Y.p, n, m, r, core.p);
      double h[2];
      if (alg == SYMPROP_HOOI) {
        // rel_residual(core_prev, core) on the unpacked cores
        dense::weighted_sq<double>(st, core_prev.p, core.p, dD.p, r, m, red.p);
        SPB_CUDA(cudaMemcpyAsync(h, red.p, sizeof(h), cudaMemcpyDeviceToHost, st));
        SPB_CUDA(cudaStreamSynchronize(st));
        rel_res = h[0] / h[1];
      } else {
        // rel_residual(factor, factor_prev)
        dense::weighted_sq<double>(st, U.p, Uprev.p, nullptr, n, r, red.p);
        SPB_CUDA(cudaMemcpyAsync(h, red.p, sizeof(h), cudaMemcpyDeviceToHost, st));
        SPB_CUDA(cudaStreamSynchronize(st));
        rel_res = h[0] / h[1];
      }
      dense::weighted_sq<double>(st, core.p, nullptr, dD.p, r, m, red.p);
      SPB_CUDA(cudaMemcpyAsync(h, red.p, sizeof(h), cudaMemcpyDeviceToHost, st));
      SPB_CUDA(cudaStreamSynchronize(st));
      cn2 = h[1];
    } else {  // HOQRI
      if (mx) {
        // core in FP64 (objective) from the FP32 Y; the update
        // U = Y diag(D) core^T (symgemm, src/dense/matrixops.cpp:102-124) as
        // (Y D^1/2)(D^1/2 core^T) on the tensor cores
        dense::core_from_f32(st, U.p, Y32.p, n, m, r, core.p);
        gram::split(st, Y32.p, sD32.p, Z);
        tc_times(core.p, (size_t)m, 1, dsD.p, U.p);
      } else {
        dense::core_from_f64(st, U.p, Y.p, n, m, r, core.p);
        dense::gemm<double>(st, n, r, m, 1.0, Y.p, m, false, core.p, m, true, 0.0, U.p, r, dD.p);
      }
      dense::orthonormalize(st, U.p, n, r);  // qr (src/dense/matrixops.cpp:58-75)
      double h[2];
      dense::weighted_sq<double>(st, core.p, core_prev.p, dD.p, r, m, red.p);
      SPB_CUDA(cudaMemcpyAsync(h, red.p, sizeof(h), cudaMemcpyDeviceToHost, st));
      SPB_CUDA(cudaStreamSynchronize(st));
      rel_res = h[0] / h[1];  // symtens_rel_res (src/dense/symtensor.cpp:78-95)
      cn2 = h[1];
    }
    dense_ms += tphase.stop_ms();
    nvtxRangePop();
    if (tc) {
      int herr = 0;
      SPB_CUDA(cudaMemcpy(&herr, gram_err.p, sizeof(int), cudaMemcpyDeviceToHost));
      if (herr) fail(SYMPROP_ERR_TIMEOUT, "tensor-core Gram: a bounded wait expired");
    }

    error = std::sqrt(normX * normX - cn2) / normX;
    if (trace) {
      std::fprintf(stderr, "tucker: iter %llu %s s3ttmc %.1f ms dense %.1f ms (iteration %.1f ms) error %.12e\n",
                   (unsigned long long)iter, mx ? "mixed" : "fp64", s3_ms - s3_prev, dense_ms - dense_prev,
                   titer.stop_ms(), error);
      s3_prev = s3_ms;
      dense_prev = dense_ms;
    }
    if (iter < res.trace_cap) {
      if (res.error_trace) res.error_trace[iter] = error;
      if (res.relres_trace) res.relres_trace[iter] = rel_res;
    }
    if (c.verbose) {
      std::cout << std::scientific << std::setprecision(prec_digits) << "Iteration: " << iter
                << " relative residual: " << rel_res << " error " << error << "\n";
    }
    iters = iter + 1;
    if (alg == SYMPROP_HOQRI) {
      SPB_CUDA(cudaMemcpyAsync(core_prev.p, core.p, sizeof(double) * r * m, cudaMemcpyDeviceToDevice, st));
    }
    double error_diff = std::abs(prev_error - error);
    const double fit = std::max(0.0, 1.0 - error * error);
    const double mixed_floor = 4.0 * fit * kMixedRel / (2.0 * std::max(error, 1e-6));
    if (mx && error_diff < std::max(c.rel_tol, mixed_floor)) {
      if (c.rel_tol >= mixed_floor) break;  // converged within the mixed resolution
      mx = false;                           // continue in FP64 from the mixed iterate
    } else if (error_diff < c.rel_tol) {
      break;
    }
    prev_error = error;
    if (alg == SYMPROP_HOOI) {
      SPB_CUDA(cudaMemcpyAsync(core_prev.p, core.p, sizeof(double) * r * m, cudaMemcpyDeviceToDevice, st));
    } else if (alg == SYMPROP_ALTHOOI) {
      SPB_CUDA(cudaMemcpyAsync(Uprev.p, U.p, sizeof(double) * n * r, cudaMemcpyDeviceToDevice, st));
    }
  }

  // outputs
  const auto wout = std::chrono::steady_clock::now();
  const size_t csize = (size_t)r * full;
  if (res.core) {
    std::vector<double> hc(csize, 0.0);
    if (alg == SYMPROP_ALTHOOI) {
      // AltHOOI writes the packed r x m core into the front of _core
      SPB_CUDA(cudaMemcpyAsync(hc.data(), core.p, sizeof(double) * r * m, cudaMemcpyDeviceToHost, st));
    } else {
      DBuf<double> cu(csize);
      unpack_rows(core.p, (uint64_t)r, (uint32_t)r, (uint32_t)L, cu.p, SYMPROP_FP64, st);
      SPB_CUDA(cudaMemcpyAsync(hc.data(), cu.p, sizeof(double) * csize, cudaMemcpyDeviceToHost, st));
      SPB_CUDA(cudaStreamSynchronize(st));
    }
    SPB_CUDA(cudaStreamSynchronize(st));
    std::copy(hc.begin(), hc.end(), res.core);
  }
  if (res.factor) {
    SPB_CUDA(cudaMemcpyAsync(res.factor, U.p, sizeof(double) * n * r, cudaMemcpyDeviceToHost, st));
  }
  SPB_CUDA(cudaStreamSynchronize(st));
  res.time_ms = tall.stop_ms();
  if (trace)
    std::fprintf(stderr, "tucker: outputs %.1f ms, total %.1f ms\n",
                 std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - wout).count(),
                 res.time_ms);
  (void)wall0;
  res.s3ttmc_ms = s3_ms;
  res.dense_ms = dense_ms;
  res.iterations = iters;
  res.error = error;
  res.core_norm = std::sqrt(cn2);
  return status;
}

// hoevd: U = top-r eigenvectors of A = X_(1) X_(1)^T built on the device
// from the leaf-grouped owners (src/sparse/spsymtensor.cpp:363-382).
void hoevd_factor(TensorState &t, cudaStream_t st, int r, double *U, bool print_matrix) {
  const int n = (int)t.dim;
  // large n: A is never formed (hoevd.cu); SPB_HOEVD_MATRIX_FREE=1 forces it
  const char *mf = std::getenv("SPB_HOEVD_MATRIX_FREE");
  if (n > kHoevdDenseMax || (mf && *mf == '1')) {
    if (hoevd_matrix_free(t, st, r, U) != SYMPROP_OK) std::printf("Eigendecomposition failed to converge.\n");
    return;
  }
  tree_build(t);
  const TreeLevels &tr = *t.tree;
  const uint32_t lv = tr.depth - 1;
  DBuf<double> A((size_t)n * n);
  SPB_CUDA(cudaMemsetAsync(A.p, 0, sizeof(double) * n * n, st));
  uint64_t nleaf = tr.size[lv];
  if (nleaf) {
    hoevd_syrk_kernel<<<(unsigned)((nleaf + 127) / 128), 128, 0, st>>>(
        tr.level_ptr[lv].p, tr.own_rem.p, tr.own_val.p, tr.leaf_mult.p, nleaf, n, A.p);
    SPB_LAUNCH_CHECK();
  }
  if (print_matrix) {
    std::vector<double> h((size_t)n * n);
    SPB_CUDA(cudaMemcpyAsync(h.data(), A.p, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, st));
    SPB_CUDA(cudaStreamSynchronize(st));
    for (int i = 0; i < n; i++) {
      for (int j = 0; j < n; j++) std::cout << h[(size_t)i * n + j] << ",";
      std::cout << "\n";
    }
  }
  std::vector<double> lam(r);
  int e = dense::top_eigs(st, A.p, n, r, U, lam.data(), nullptr, 1e-12, 100);
  if (e != SYMPROP_OK) std::printf("Eigendecomposition failed to converge.\n");
}

}  // namespace spb

extern "C" int symprop_tucker(const symprop_tensor *t, const symprop_config *cfg, int alg,
                              symprop_result *res) {
  int st = SYMPROP_OK;
  int g = spb::guard([&] {
    if (!t || !cfg || !res) spb::fail(SYMPROP_ERR_INVALID, "null argument");
    SPB_CUDA(cudaSetDevice(t->s.device));
    st = spb::run_tucker(const_cast<spb::TensorState &>(t->s), *cfg, alg, *res);
  });
  if (g != SYMPROP_OK) return g;
  if (st != SYMPROP_OK) {
    spb::set_last_error("eigensolver did not reach its tolerance (results returned)");
  }
  return st;
}
