// extern "C" host-pointer forms of the reference's symprop::matrix
// operations (include/detail/dense/matrixops.hpp:12-45,
// src/dense/matrixops.cpp:18-146), run on the current device with the FP64
// building blocks of dense.cu in place of CBLAS/LAPACKE:
//   gemmtn   C = A^T B                       dense::gemm (transA)
//   symgemm  C = A diag(c) B^T               dense::gemm (transB, k-scale)
//   symsyrk  upper(C) = A diag(c) A^T        dense::gemm (symmetric)
//   qr       explicit Householder Q          dense::householder_q
//   syevd    top eigenvectors, ascending     dense::top_eigs / jacobi_eig
//   leftsvd  leading left singular vectors   eigenvectors of the smaller Gram
// Operands are copied in, the result copied out; every call synchronises.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "dense.cuh"

using namespace spb;

namespace {

void require(bool ok, const char *what) {
  if (!ok) fail(SYMPROP_ERR_INVALID, "%s", what);
}

void require_device() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    fail(SYMPROP_ERR_NODEVICE, "no CUDA device visible");
  }
}

// dense::gemm takes int sizes and leading dimensions
void require_int(uint64_t v, const char *what) {
  if (v >= (1ull << 31)) fail(SYMPROP_ERR_SIZE, "%s = %llu does not fit the device GEMM", what,
                              (unsigned long long)v);
}

void to_device(DBuf<double> &d, const double *h, uint64_t n) {
  d.alloc(n);
  if (n) SPB_CUDA(cudaMemcpy(d.p, h, n * sizeof(double), cudaMemcpyHostToDevice));
}

void to_host(double *h, const DBuf<double> &d, uint64_t n) {
  if (n) SPB_CUDA(cudaMemcpy(h, d.p, n * sizeof(double), cudaMemcpyDeviceToHost));
}

// V (s x r) = top-r eigenvectors of the device matrix S (s x s), descending.
// Returns SYMPROP_ERR_NOCONV (V then holds the last iterate) if the
// residual did not reach 1e-12 of the largest eigenvalue.
int top_eigvecs(const double *S, int s, int r, double *V) {
  std::vector<double> lam((size_t)r);
  return dense::top_eigs(0, S, s, r, V, lam.data(), nullptr, 1e-12, 200);
}

void fail_noconv(int st, const char *what) {
  if (st != SYMPROP_OK) fail(st, "%s: eigensolver did not converge (the result holds its last iterate)", what);
}

__global__ void reverse_cols_kernel(const double *V, int rows, int r, double *U) {
  const size_t n = (size_t)rows * r;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const size_t row = i / r;
    const int j = (int)(i - row * r);
    U[i] = V[row * r + (r - 1 - j)];
  }
}

unsigned grid_for(uint64_t n) { return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, 148 * 32)); }

}  // namespace

extern "C" {

int symprop_gemmtn(double *C, const double *A, const double *B, uint64_t arow, uint64_t acol,
                   uint64_t bcol) {
  return guard([&] {
    require(C && (arow == 0 || ((A || !acol) && (B || !bcol))), "null argument");
    require_int(arow, "arow");
    require_int(acol, "acol");
    require_int(bcol, "bcol");
    if (!acol || !bcol) return;
    require_device();
    DBuf<double> dA, dB, dC(acol * bcol);
    to_device(dA, A, arow * acol);
    to_device(dB, B, arow * bcol);
    dense::gemm<double>(0, (int)acol, (int)bcol, (int)arow, 1.0, dA.p, (int)acol, true, dB.p, (int)bcol, false, 0.0,
                        dC.p, (int)bcol);
    to_host(C, dC, acol * bcol);
  });
}

int symprop_symgemm(double *C, const double *A, const double *B, const double *row_coeff,
                    uint64_t ncoeff, uint64_t I1, uint64_t I2) {
  return guard([&] {
    require(C && (ncoeff == 0 || (row_coeff && (A || !I1) && (B || !I2))), "null argument");
    require_int(ncoeff, "ncoeff");
    require_int(I1, "I1");
    require_int(I2, "I2");
    if (!I1 || !I2) return;
    require_device();
    DBuf<double> dA, dB, dc, dC(I1 * I2);
    to_device(dA, A, I1 * ncoeff);
    to_device(dB, B, I2 * ncoeff);
    to_device(dc, row_coeff, ncoeff);
    dense::gemm<double>(0, (int)I1, (int)I2, (int)ncoeff, 1.0, dA.p, (int)ncoeff, false, dB.p, (int)ncoeff, true, 0.0,
                        dC.p, (int)I2, dc.p);
    to_host(C, dC, I1 * I2);
  });
}

int symprop_symsyrk(double *C, const double *A, const double *row_coeff, uint64_t ncoeff,
                    uint64_t I1) {
  return guard([&] {
    require(C && (ncoeff == 0 || (row_coeff && (A || !I1))), "null argument");
    require_int(ncoeff, "ncoeff");
    require_int(I1, "I1");
    if (!I1) return;
    require_device();
    DBuf<double> dA, dc, dC(I1 * I1);
    to_device(dA, A, I1 * ncoeff);
    to_device(dc, row_coeff, ncoeff);
    dense::gemm<double>(0, (int)I1, (int)I1, (int)ncoeff, 1.0, dA.p, (int)ncoeff, false, dA.p, (int)ncoeff, true, 0.0,
                        dC.p, (int)I1, dc.p, true);
    // rows i, columns i..I1-1 only (the upper triangle cblas_dsyrk writes),
    // through a host block of at most 64 MiB
    const uint64_t rows_per = std::max<uint64_t>(1, (64ull << 20) / (I1 * sizeof(double)));
    std::vector<double> blk(std::min(I1, rows_per) * I1);
    for (uint64_t r0 = 0; r0 < I1; r0 += rows_per) {
      const uint64_t r1 = std::min(I1, r0 + rows_per);
      SPB_CUDA(cudaMemcpy(blk.data(), dC.p + r0 * I1, (r1 - r0) * I1 * sizeof(double), cudaMemcpyDeviceToHost));
      for (uint64_t i = r0; i < r1; ++i)
        std::memcpy(C + i * I1 + i, blk.data() + (i - r0) * I1 + i, (I1 - i) * sizeof(double));
    }
  });
}

int symprop_qr(double *A, uint64_t nr, uint64_t nc) {
  return guard([&] {
    require(A || !nr || !nc, "null argument");
    require(nr >= nc, "qr needs nr >= nc");
    require_int(nr * nc, "nr * nc");
    if (!nc) return;
    require_device();
    DBuf<double> dA;
    to_device(dA, A, nr * nc);
    dense::householder_q(0, dA.p, (int)nr, (int)nc);
    to_host(A, dA, nr * nc);
  });
}

int symprop_syevd(const double *A, double *U, uint64_t dim, uint64_t rank) {
  return guard([&] {
    require(A && U, "null argument");
    require(rank >= 1 && rank <= dim, "rank must be in [1, dim]");
    require_int(dim * dim, "dim * dim");
    require_device();
    DBuf<double> dA, dV(dim * rank), dU(dim * rank);
    to_device(dA, A, dim * dim);
    const int st = top_eigvecs(dA.p, (int)dim, (int)rank, dV.p);
    reverse_cols_kernel<<<grid_for(dim * rank), 256>>>(dV.p, (int)dim, (int)rank, dU.p);
    SPB_LAUNCH_CHECK();
    to_host(U, dU, dim * rank);
    fail_noconv(st, "syevd");
  });
}

int symprop_leftsvd(const double *A, double *U, uint64_t nr, uint64_t nc, uint64_t rank) {
  return guard([&] {
    require(A && U, "null argument");
    require(rank >= 1 && rank <= std::min(nr, nc), "rank must be in [1, min(nr, nc)]");
    require_int(nr * nc, "nr * nc");
    require_device();
    DBuf<double> dA, dU(nr * rank);
    to_device(dA, A, nr * nc);
    int st = SYMPROP_OK;
    if (nr <= nc) {
      // U = top eigenvectors of A A^T (nr x nr)
      DBuf<double> G(nr * nr);
      dense::gemm<double>(0, (int)nr, (int)nr, (int)nc, 1.0, dA.p, (int)nc, false, dA.p, (int)nc, true, 0.0, G.p,
                          (int)nr, nullptr, true);
      st = top_eigvecs(G.p, (int)nr, (int)rank, dU.p);
    } else {
      // V = top eigenvectors of A^T A (nc x nc); U = A V, columns normalised
      // (they are orthogonal with norms sigma_j; CholQR keeps each column's
      // direction)
      DBuf<double> G(nc * nc), V(nc * rank);
      dense::gemm<double>(0, (int)nc, (int)nc, (int)nr, 1.0, dA.p, (int)nc, true, dA.p, (int)nc, false, 0.0, G.p,
                          (int)nc, nullptr, true);
      st = top_eigvecs(G.p, (int)nc, (int)rank, V.p);
      dense::gemm<double>(0, (int)nr, (int)rank, (int)nc, 1.0, dA.p, (int)nc, false, V.p, (int)rank, false, 0.0,
                          dU.p, (int)rank);
      dense::orthonormalize(0, dU.p, (int)nr, (int)rank);
    }
    to_host(U, dU, nr * rank);
    fail_noconv(st, "leftsvd");
  });
}

}  // extern "C"
