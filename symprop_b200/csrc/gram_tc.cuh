// tcgen05 split-BF16 Gram matrix (gram_tc.cu).
#pragma once

#include "common.cuh"

namespace spb {
namespace gram {

// bytes of workspace gram_split_bf16 needs for an n x m input
size_t workspace_bytes(int n, int m);

// S (m x m, FP64, full symmetric) = (Y diag(sd))^T (Y diag(sd)) from an
// FP32 row-major n x m Y, on the tensor cores (BF16 hi/lo split, FP32
// accumulation).  *d_err is set to 1 if a bounded wait expired.
void gram_split_bf16(cudaStream_t st, const float *Y, int n, int m, const float *sd, double *S,
                     void *ws, int *d_err);

}  // namespace gram
}  // namespace spb
