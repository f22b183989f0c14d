// Dense FP64/FP32 building blocks of the Tucker loop (dense.cu):
// tiled GEMM with deterministic split-K, weighted reductions, orthonormal
// bases (CholQR2 with a Householder fallback), a one-CTA Jacobi eigensolver
// and a block-Krylov top-r symmetric eigensolver.  They replace the
// CBLAS/LAPACKE calls of the reference (src/dense/matrixops.cpp:18-146).
#pragma once

#include <functional>

#include "common.cuh"

namespace spb {
namespace dense {

// C[M x N] = alpha * sum_k a(i,k) b(k,j) (kscale ? kscale[k] : 1) + beta * C
//   a(i,k) = transA ? A[k*lda + i] : A[i*lda + k]
//   b(k,j) = transB ? B[j*ldb + k] : B[k*ldb + j]
// sym_upper: only the upper triangle is computed and mirrored (M == N, C symmetric).
template <typename T>
void gemm(cudaStream_t st, int M, int N, int K, T alpha, const T *A, int lda, bool transA,
          const T *B, int ldb, bool transB, T beta, T *C, int ldc, const T *kscale = nullptr,
          bool sym_upper = false);

// core (r x m, FP64) = U^T Y for FP64 U (n x r) and FP32 Y (n x m), both
// row-major: Y is read once and widened in registers, FP64 accumulation,
// deterministic (fixed row chunks summed in order).
void core_from_f32(cudaStream_t st, const double *U, const float *Y, int n, int m, int r, double *core);
// the same r x m core U^T Y from an FP64 Y (one read of Y, fixed-order FP64 sums)
void core_from_f64(cudaStream_t st, const double *U, const double *Y, int n, int m, int r, double *core);

// sum_{i<rows, q<cols} w[q] * (X[i,q] - (Y ? Y[i,q] : 0))^2 and sum w X^2 (FP64 out, deterministic)
template <typename T>
void weighted_sq(cudaStream_t st, const T *X, const T *Y, const double *w, int rows, int cols,
                 double *d_out2);

// Orthonormal basis of the columns of A (rows x cols, row-major, in place).
// CholQR2; a Householder QR replaces it when the Gram matrix is numerically
// singular.  Returns true if the Householder path was used.
bool orthonormalize(cudaStream_t st, double *A, int rows, int cols);

// Householder QR: A (rows x cols) replaced by the explicit Q of dgeqrf+dorgqr.
void householder_q(cudaStream_t st, double *A, int rows, int cols);

// Symmetric eigendecomposition of a small matrix (n <= kJacobiMax) in one CTA:
// eigenvalues descending in w, eigenvectors as columns of V (n x n).
constexpr int kJacobiMax = 96;
void jacobi_eig(cudaStream_t st, const double *S, int n, double *w, double *V);

// Top-r eigenpairs of a symmetric s x s matrix S (device, FP64).  V (s x r)
// receives orthonormal eigenvectors, lam (host) the eigenvalues in
// descending order.  warm (s x r) may hold a starting subspace.
// Returns SYMPROP_OK or SYMPROP_ERR_NOCONV.
int top_eigs(cudaStream_t st, const double *S, int s, int r, double *V, double *lam,
             const double *warm, double tol, int max_restarts);

// The same for a symmetric operator given by its action Y = S X on row-major
// blocks (X: s x cols with leading dimension ldx, Y: s x cols, ldy), for
// matrices that are never formed.
using SymApply = std::function<void(cudaStream_t st, const double *X, int ldx, int cols, double *Y, int ldy)>;
int top_eigs_op(cudaStream_t st, const SymApply &apply, int s, int r, double *V, double *lam,
                const double *warm, double tol, int max_restarts);

// elementwise helpers
void scale_sym(cudaStream_t st, double *G, int m, const double *sd);  // G[i][j] *= sd[i] sd[j]
void scale_rows_clip(cudaStream_t st, double *U, int n, int r, double delta);
template <typename Ts, typename Td> void convert(cudaStream_t st, const Ts *src, Td *dst, size_t n);

}  // namespace dense
}  // namespace spb
