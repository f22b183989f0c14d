// hoevd initialisation (src/sparse/spsymtensor.cpp:363-439): U = the top-r
// eigenvectors of A = X_(1) X_(1)^T.
//
// The reference forms A from a COO list of every distinct permutation of
// every nonzero (sparse_syrk, :385-409); its column key is a base-n number
// of N-1 ids, which overflows 64 bits once n^(N-1) >= 2^64, and A itself is
// n x n dense (320 GB at n = 200k).  Here A is grouped by the tree's leaves
// C (the unique (N-1)-sub-multisets, each with its distinct owners
// (row p, value x_p) and its permutation count mult(C)):
//     A = sum_C mult(C) w_C w_C^T,   w_C = sum_p x_p e_p,
// so the eigensolver only needs the action
//     A X = sum_C mult(C) w_C (w_C^T X):
// one pass gathers z_C = w_C^T X per leaf, a second pass adds
// mult(C) x_p z_C into row p from a row-sorted copy of the owners
// (segmented sum, no atomics).  Small n keeps the dense A of tucker.cu.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstdlib>
#include <vector>

#include "dense.cuh"
#include "tensor.cuh"

namespace spb {
namespace {

// grid-stride kernels: at most 148 x 64 blocks
inline unsigned blocks_for(uint64_t n, unsigned block) {
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + block - 1) / block, 148u * 64u));
}

// owner i is kept when it is the first of its leaf or its row differs from
// the previous owner's (repeated ids give adjacent duplicate owners)
__global__ void distinct_kernel(const uint64_t *own_ptr, uint64_t nleaf, const uint64_t *rem, uint32_t *leaf_of,
                                uint8_t *keep) {
  for (uint64_t leaf = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; leaf < nleaf;
       leaf += (uint64_t)gridDim.x * blockDim.x)
    for (uint64_t i = own_ptr[leaf]; i < own_ptr[leaf + 1]; ++i) {
      leaf_of[i] = (uint32_t)leaf;
      keep[i] = (i == own_ptr[leaf] || rem[i] != rem[i - 1]) ? 1 : 0;
    }
}

__global__ void row_keys_kernel(const uint64_t *rem, const uint8_t *keep, uint64_t nown, uint32_t dim,
                                uint32_t *key, uint32_t *idx) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nown;
       i += (uint64_t)gridDim.x * blockDim.x) {
    key[i] = keep[i] ? (uint32_t)(rem[i] - 1) : dim;  // dropped owners sort past the last row
    idx[i] = (uint32_t)i;
  }
}

__global__ void row_ptr_kernel(const uint32_t *rows_sorted, uint64_t n, uint32_t dim, uint64_t *row_ptr) {
  for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r <= dim;
       r += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t lo = 0, hi = n;
    while (lo < hi) {
      const uint64_t mid = (lo + hi) >> 1;
      if (rows_sorted[mid] < r) lo = mid + 1; else hi = mid;
    }
    row_ptr[r] = lo;
  }
}

// z[leaf][c] = sum over the leaf's distinct owners of x * X[row][c0 + c]
__global__ void gather_kernel(const uint64_t *own_ptr, uint64_t nleaf, const uint64_t *rem, const double *val,
                              const uint8_t *keep, const double *X, int ldx, int c0, int cols, double *Z) {
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nleaf * (uint64_t)cols;
       t += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t leaf = t / (uint64_t)cols;
    const int c = (int)(t - leaf * (uint64_t)cols);
    double z = 0.0;
    for (uint64_t i = own_ptr[leaf]; i < own_ptr[leaf + 1]; ++i)
      if (keep[i]) z += val[i] * X[(rem[i] - 1) * (uint64_t)ldx + c0 + c];
    Z[t] = z;
  }
}

// Y[row][c0 + c] = sum over the row's owners of mult(leaf) * x * z[leaf][c]
__global__ void scatter_kernel(const uint64_t *row_ptr, uint32_t dim, const uint32_t *owner_sorted,
                               const uint32_t *leaf_of, const double *val, const double *mult, const double *Z,
                               int cols, int c0, double *Y, int ldy) {
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < (uint64_t)dim * cols;
       t += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t row = t / (uint64_t)cols;
    const int c = (int)(t - row * (uint64_t)cols);
    double y = 0.0;
    for (uint64_t e = row_ptr[row]; e < row_ptr[row + 1]; ++e) {
      const uint32_t i = owner_sorted[e], leaf = leaf_of[i];
      y += mult[leaf] * val[i] * Z[(uint64_t)leaf * cols + c];
    }
    Y[row * (uint64_t)ldy + c0 + c] = y;
  }
}

}  // namespace

// Top-r eigenvectors of A = X_(1) X_(1)^T without forming A (see above).
// U: n x r device, row-major.  Returns the eigensolver status.
int hoevd_matrix_free(TensorState &t, cudaStream_t st, int r, double *U) {
  NvtxRange nv("hoevd (matrix-free)");
  tree_build(t);
  const TreeLevels &tr = *t.tree;
  const uint32_t lv = tr.depth - 1;
  const uint64_t nleaf = tr.size[lv], nown = tr.nown;
  const uint32_t n = t.dim;
  if (nown >= (1ull << 32)) fail(SYMPROP_ERR_SIZE, "hoevd: more than 2^32 owners");
  const uint64_t *own_ptr = tr.level_ptr[lv].p;
  DBuf<uint32_t> leaf_of(std::max<uint64_t>(nown, 1));
  DBuf<uint8_t> keep(std::max<uint64_t>(nown, 1));
  DBuf<uint32_t> key(std::max<uint64_t>(nown, 1)), key_sorted(std::max<uint64_t>(nown, 1));
  DBuf<uint32_t> idx(std::max<uint64_t>(nown, 1)), owner_sorted(std::max<uint64_t>(nown, 1));
  DBuf<uint64_t> row_ptr((uint64_t)n + 1);
  if (nleaf) {
    distinct_kernel<<<blocks_for(nleaf, 256), 256, 0, st>>>(own_ptr, nleaf, tr.own_rem.p, leaf_of.p, keep.p);
    SPB_LAUNCH_CHECK();
  }
  if (nown) {
    row_keys_kernel<<<blocks_for(nown, 256), 256, 0, st>>>(tr.own_rem.p, keep.p, nown, n, key.p, idx.p);
    SPB_LAUNCH_CHECK();
    int bits = 1;
    while (bits < 32 && (1ull << bits) <= n) ++bits;
    size_t tmp = 0;
    SPB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, key.p, key_sorted.p, idx.p, owner_sorted.p,
                                             (int64_t)nown, 0, bits, st));
    DBuf<char> work(std::max<size_t>(tmp, 1));
    SPB_CUDA(cub::DeviceRadixSort::SortPairs(work.p, tmp, key.p, key_sorted.p, idx.p, owner_sorted.p,
                                             (int64_t)nown, 0, bits, st));
  }
  row_ptr_kernel<<<blocks_for((uint64_t)n + 1, 256), 256, 0, st>>>(key_sorted.p, nown, n, row_ptr.p);
  SPB_LAUNCH_CHECK();
  key.release();
  idx.release();
  // columns per pass: the leaf block z stays within about 4 GiB
  const uint64_t budget = 4ull << 30;
  const int chunk = (int)std::max<uint64_t>(1, std::min<uint64_t>(32, budget / (std::max<uint64_t>(nleaf, 1) * 8)));
  DBuf<double> Z(std::max<uint64_t>(nleaf, 1) * chunk);
  const uint64_t *rem = tr.own_rem.p;
  const double *val = tr.own_val.p, *mult = tr.leaf_mult.p;
  dense::SymApply apply = [&](cudaStream_t s, const double *X, int ldx, int cols, double *Y, int ldy) {
    for (int c0 = 0; c0 < cols; c0 += chunk) {
      const int cc = std::min(chunk, cols - c0);
      if (nleaf) {
        gather_kernel<<<blocks_for(nleaf * cc, 256), 256, 0, s>>>(own_ptr, nleaf, rem, val, keep.p, X, ldx, c0, cc,
                                                                  Z.p);
        SPB_LAUNCH_CHECK();
      }
      scatter_kernel<<<blocks_for((uint64_t)n * cc, 256), 256, 0, s>>>(row_ptr.p, n, owner_sorted.p, leaf_of.p, val,
                                                                       mult, Z.p, cc, c0, Y, ldy);
      SPB_LAUNCH_CHECK();
    }
  };
  std::vector<double> lam(r);
  return dense::top_eigs_op(st, apply, (int)n, r, U, lam.data(), nullptr, 1e-12, 100);
}

}  // namespace spb
