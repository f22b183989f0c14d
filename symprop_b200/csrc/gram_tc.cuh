// Mixed-precision dense products on the tcgen05 tensor cores (gram_tc.cu):
// split-BF16 operands, FP32 accumulation.
#pragma once

#include <cuda_bf16.h>

#include "common.cuh"

namespace spb {
namespace gram {

// Rows of the panel P in W = Z P^T (UMMA N = 16): r <= kPanelRows.
constexpr int kPanelRows = 16;

// Z = X diag(colscale) held as Z ~ H + L (H = bf16(Z), L = bf16(Z - H)),
// row-major rows x ld, ld = cols rounded up to 64 (zero padded).
struct Split {
  __nv_bfloat16 *h = nullptr, *l = nullptr;
  int rows = 0, cols = 0, ld = 0;
};

int split_ld(int cols);
size_t split_bytes(int rows, int cols);
// H and L views of a workspace of split_bytes(rows, cols) bytes
Split split_view(void *ws, int rows, int cols);
// fills z from the FP32 row-major rows x cols X (colscale may be null)
void split(cudaStream_t st, const float *X, const float *colscale, const Split &z);

// S (full symmetric FP64) = Z^T Z (cols x cols) or Z Z^T (rows x rows),
// from the upper tiles, the K axis cut into splits whose FP32 partial sums
// are added in FP64; scratch of gram_cols_scratch_bytes(rows, cols) /
// gram_rows_scratch_bytes(rows, cols) bytes.  *d_err is set to 1 if a
// bounded wait expired.
size_t gram_cols_scratch_bytes(int rows, int cols);
size_t gram_rows_scratch_bytes(int rows, int cols);
void gram_cols(cudaStream_t st, const Split &z, double *S, void *scratch, int *d_err);
void gram_rows(cudaStream_t st, const Split &z, double *S, void *scratch, int *d_err);

// W (rows x r FP64, row stride ldw) = Z P^T with P[q][k] = P[q * sq + k * sk]
// * colscale[k] (colscale may be null), q < r <= kPanelRows, k < cols;
// scratch of times_scratch_bytes(rows, cols) bytes.
size_t times_scratch_bytes(int rows, int cols);
void times(cudaStream_t st, const Split &z, const double *P, int r, size_t sq, size_t sk,
           const double *colscale, double *W, size_t ldw, void *scratch, int *d_err);

// S (m x m) = (Y diag(sd))^T (Y diag(sd)) from an FP32 row-major n x m Y:
// the split and the column Gram in a workspace of workspace_bytes(n, m).
size_t workspace_bytes(int n, int m);
void gram_split_bf16(cudaStream_t st, const float *Y, int n, int m, const float *sd, double *S,
                     void *ws, int *d_err);

// bound of the tensor-core kernels' main-loop waits (failure-injection hook)
uint64_t mainloop_wait_ns();
void set_mainloop_wait_ns(uint64_t ns);

}  // namespace gram
}  // namespace spb
