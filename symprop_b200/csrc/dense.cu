// Dense steps of the Tucker loop on sm_100a (FP64 drop-in precision).
//
// Replaces the reference's CBLAS/LAPACKE wrappers
// (src/dense/matrixops.cpp): gemmtn (:45-56), symgemm (:102-124) and
// symsyrk (:126-146) become the tiled GEMM below; leftsvd (:18-43) and
// syevd (:77-100) become a block-Krylov top-r eigensolver on the packed Gram
// matrix with a one-CTA Jacobi for the projected problem; qr (:58-75)
// becomes CholQR2 with a Householder QR fallback.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdint>
#include <cstdlib>
#include <map>
#include <mutex>
#include <type_traits>
#include <vector>

#include "dense.cuh"

namespace spb {
namespace dense {

namespace {

inline unsigned cdiv(long long a, long long b) { return (unsigned)((a + b - 1) / b); }

// ------------------------------------------------------------------- GEMM

constexpr int BM = 64, BN = 64, BK = 16;

template <typename T, bool TA, bool TB, bool KS>
__global__ void __launch_bounds__(256) gemm_tile_kernel(int M, int N, int K, const T *__restrict__ A,
                                                        int lda, const T *__restrict__ B, int ldb,
                                                        const T *__restrict__ ks, T *out, int ldo,
                                                        int kchunk, int sym_upper,
                                                        size_t split_stride) {
  const int tm = blockIdx.y, tn = blockIdx.x;
  if (sym_upper && tm > tn) return;
  const int bm = tm * BM, bn = tn * BN;
  const int k0 = blockIdx.z * kchunk;
  const int k1 = min(K, k0 + kchunk);
  __shared__ T As[BK][BM + 1];
  __shared__ T Bs[BK][BN + 1];
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  T acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = T(0);
  for (int kk = k0; kk < k1; kk += BK) {
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      int idx = tid + e * 256;
      int kq, im;
      if (TA) { kq = idx / BM; im = idx % BM; } else { im = idx / BK; kq = idx % BK; }
      int gi = bm + im, gk = kk + kq;
      T v = T(0);
      if (gi < M && gk < k1) {
        v = TA ? A[(size_t)gk * lda + gi] : A[(size_t)gi * lda + gk];
        if (KS) v *= ks[gk];
      }
      As[kq][im] = v;
      int jn;
      if (TB) { jn = idx / BK; kq = idx % BK; } else { kq = idx / BN; jn = idx % BN; }
      int gj = bn + jn;
      gk = kk + kq;
      T w = T(0);
      if (gj < N && gk < k1) w = TB ? B[(size_t)gj * ldb + gk] : B[(size_t)gk * ldb + gj];
      Bs[kq][jn] = w;
    }
    __syncthreads();
#pragma unroll
    for (int kq = 0; kq < BK; ++kq) {
      T a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kq][ty * 4 + i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[kq][tx * 4 + j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] += a[i] * b[j];
    }
    __syncthreads();
  }
  T *o = out + blockIdx.z * split_stride;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    int gi = bm + ty * 4 + i;
    if (gi >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      int gj = bn + tx * 4 + j;
      if (gj < N) o[(size_t)gi * ldo + gj] = acc[i][j];
    }
  }
}

// ------------------------------------------------ FP64 Gram C = A^T A
//
// The m x m Gram of the columns of a row-major n x m matrix (HOOI's dense
// step in FP64), upper tiles only: 128 x 128 tiles of C, 256 threads with
// 8 x 8 accumulators each (rows 32 q + 2 ty + {0, 1}, q < 4, the same for
// the columns with tx: a warp's 16-byte loads of one k row are then
// contiguous and free of bank conflicts), k-blocks of 16 rows of A staged in shared
// memory by cp.async in a 3-stage ring.  The K axis is cut into splits
// whose partial tiles the finalize kernel adds (and mirrors).
constexpr int GB = 128, GK = 16, GST = 3;

struct GramSmem {
  double a[GST][GK][GB];
  double b[GST][GK][GB];
};

__device__ __forceinline__ void cp_async16_zfill(void *dst, const void *src, bool full) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  const int sz = full ? 16 : 0;  // 0: fill the 16 bytes with zeros, read nothing
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(sz) : "memory");
}

__global__ void __launch_bounds__(256, 1) gram_tn_f64_kernel(int M, int K, const double *__restrict__ A, int lda,
                                                             int ntile, int kchunk, double *out,
                                                             size_t split_stride) {
  extern __shared__ __align__(16) unsigned char gram_raw[];
  GramSmem &sm = *reinterpret_cast<GramSmem *>(gram_raw);
  // upper tile (ti, tj), ti <= tj, of linear index blockIdx.x (row by row)
  int ti = 0, rem = (int)blockIdx.x;
  while (rem >= ntile - ti) {
    rem -= ntile - ti;
    ++ti;
  }
  const int tj = ti + rem;
  const bool diag = ti == tj;
  const int i0 = ti * GB, j0 = tj * GB;
  const int k0 = (int)blockIdx.y * kchunk, k1 = min(K, k0 + kchunk);
  const int nkb = (k1 - k0 + GK - 1) / GK;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;

  auto load = [&](int kb, int stage) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int c = tid + 256 * q, kr = c >> 6, col = (c & 63) * 2;
      const int gk = k0 + kb * GK + kr;
      const bool oka = gk < k1 && i0 + col < M;
      cp_async16_zfill(&sm.a[stage][kr][col], oka ? A + (size_t)gk * lda + i0 + col : A, oka);
      if (!diag) {
        const bool okb = gk < k1 && j0 + col < M;
        cp_async16_zfill(&sm.b[stage][kr][col], okb ? A + (size_t)gk * lda + j0 + col : A, okb);
      }
    }
  };
#pragma unroll
  for (int s = 0; s < GST - 1; ++s) {
    if (s < nkb) load(s, s);
    asm volatile("cp.async.commit_group;" ::: "memory");
  }
  double acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = 0.0;
  for (int kb = 0; kb < nkb; ++kb) {
    asm volatile("cp.async.wait_group %0;" ::"n"(GST - 2) : "memory");
    __syncthreads();
    if (kb + GST - 1 < nkb) load(kb + GST - 1, (kb + GST - 1) % GST);
    asm volatile("cp.async.commit_group;" ::: "memory");
    const int stg = kb % GST;
    const double(*As)[GB] = sm.a[stg];
    const double(*Bs)[GB] = diag ? sm.a[stg] : sm.b[stg];
#pragma unroll 4
    for (int kk = 0; kk < GK; ++kk) {
      double a[8], b[8];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const double2 av = *reinterpret_cast<const double2 *>(&As[kk][32 * q + 2 * ty]);
        const double2 bv = *reinterpret_cast<const double2 *>(&Bs[kk][32 * q + 2 * tx]);
        a[2 * q] = av.x, a[2 * q + 1] = av.y;
        b[2 * q] = bv.x, b[2 * q + 1] = bv.y;
      }
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  double *o = out + blockIdx.y * split_stride;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int gi = i0 + 32 * (i >> 1) + 2 * ty + (i & 1);
    if (gi >= M) continue;
#pragma unroll
    for (int jh = 0; jh < 4; ++jh) {
      const int gj = j0 + 32 * jh + 2 * tx;
      if (gj < M) *reinterpret_cast<double2 *>(&o[(size_t)gi * M + gj]) = make_double2(acc[i][2 * jh], acc[i][2 * jh + 1]);
    }
  }
}

// ------------------------------------ FP64 panel W = A diag(ks) B, N <= 16
//
// HOOI's U = Y D^1/2 V and HOQRI's Y D C^T in FP64: a tall row-major A
// (M x K) times a K x N matrix with N <= 16.  One CTA of 256 threads per 64
// rows of A, K in blocks of 32 (the A block read once, coalesced along k;
// the scaled B block broadcast from shared memory); each thread keeps 4
// outputs (row tid / 4, columns 4 (tid % 4) .. + 3).  HBM-bound on A.
constexpr int PR = 64, PK = 32;

__global__ void __launch_bounds__(256) panel_f64_kernel(int M, int N, int K, const double *__restrict__ A, int lda,
                                                        const double *__restrict__ B, int ldb, bool transB,
                                                        const double *__restrict__ ks, double *__restrict__ W,
                                                        int ldw) {
  __shared__ double As[PR][PK + 1];
  __shared__ __align__(16) double Bs[PK][16];
  const int tid = threadIdx.x, row = tid >> 2, c0 = (tid & 3) * 4;
  const int i0 = blockIdx.x * PR;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int k0 = 0; k0 < K; k0 += PK) {
    double av[PR * PK / 256];
#pragma unroll
    for (int t = 0; t < PR * PK / 256; ++t) {
      const int e = tid + 256 * t, ii = e / PK, kk = e % PK, gi = i0 + ii, gk = k0 + kk;
      av[t] = gi < M && gk < K ? A[(size_t)gi * lda + gk] : 0.0;
    }
#pragma unroll
    for (int t = 0; t < PR * PK / 256; ++t) {
      const int e = tid + 256 * t;
      As[e / PK][e % PK] = av[t];
    }
    for (int e = tid; e < PK * 16; e += 256) {
      const int kk = e >> 4, q = e & 15, gk = k0 + kk;
      double b = 0.0;
      if (gk < K && q < N) {
        b = transB ? B[(size_t)q * ldb + gk] : B[(size_t)gk * ldb + q];
        if (ks) b *= ks[gk];
      }
      Bs[kk][q] = b;
    }
    __syncthreads();
#pragma unroll 8
    for (int kk = 0; kk < PK; ++kk) {
      const double a = As[row][kk];
      const double2 b0 = *reinterpret_cast<const double2 *>(&Bs[kk][c0]);
      const double2 b1 = *reinterpret_cast<const double2 *>(&Bs[kk][c0 + 2]);
      acc[0] = fma(a, b0.x, acc[0]);
      acc[1] = fma(a, b0.y, acc[1]);
      acc[2] = fma(a, b1.x, acc[2]);
      acc[3] = fma(a, b1.y, acc[3]);
    }
    __syncthreads();
  }
  const int gi = i0 + row;
  if (gi < M)
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if (c0 + j < N) W[(size_t)gi * ldw + c0 + j] = acc[j];
}

// C = alpha * sum_z P[z] + beta * C, mirroring the lower triangle for sym_upper
template <typename T>
__global__ void gemm_finalize_kernel(int M, int N, const T *P, int splits, size_t stride, T alpha,
                                     T beta, T *C, int ldc, int sym_upper) {
  size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (size_t)M * N) return;
  int i = (int)(idx / N), j = (int)(idx % N);
  int si = i, sj = j;
  if (sym_upper && (i / BM) > (j / BM)) { si = j; sj = i; }
  T s = T(0);
  for (int z = 0; z < splits; ++z) s += P[z * stride + (size_t)si * N + sj];
  T prev = beta != T(0) ? C[(size_t)i * ldc + j] : T(0);
  C[(size_t)i * ldc + j] = alpha * s + beta * prev;
}

// --------------------------------------------------------- reductions

constexpr int kRedBlocks = 296;

template <typename T>
__global__ void wsq_partial_kernel(const T *X, const T *Y, const double *w, int rows, int cols,
                                   double *part) {
  double a = 0.0, b = 0.0;
  size_t total = (size_t)rows * cols;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    int q = (int)(idx % cols);
    double x = (double)X[idx];
    double d = x - (Y ? (double)Y[idx] : 0.0);
    double ww = w ? w[q] : 1.0;
    a += ww * d * d;
    b += ww * x * x;
  }
  __shared__ double sa[256], sb[256];
  sa[threadIdx.x] = a;
  sb[threadIdx.x] = b;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      sa[threadIdx.x] += sa[threadIdx.x + s];
      sb[threadIdx.x] += sb[threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = sa[0];
    part[2 * blockIdx.x + 1] = sb[0];
  }
}

__global__ void sum_pairs_kernel(const double *part, int n, double *out) {
  __shared__ double sa[256], sb[256];
  double a = 0, b = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    a += part[2 * i];
    b += part[2 * i + 1];
  }
  sa[threadIdx.x] = a;
  sb[threadIdx.x] = b;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      sa[threadIdx.x] += sa[threadIdx.x + s];
      sb[threadIdx.x] += sb[threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[0] = sa[0];
    out[1] = sb[0];
  }
}

// ------------------------------------------------------------ Cholesky

// G (c x c) -> Rinv with A Rinv orthonormal for G = A^T A.  The columns are
// first scaled to unit norm (G' = D G D, D = diag(G)^-1/2), so the pivot test
// measures linear dependence, not column scaling; Rinv = D R'^-1 with
// G' = R'^T R'.  status[0] = 1 when a pivot is not safely positive.
__global__ void chol_inv_kernel(const double *G, int c, double *Rinv, int *status) {
  extern __shared__ double sm[];
  double *R = sm;          // c x c
  double *Ri = sm + c * c; // c x c
  __shared__ double dsc[64];
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int i = tid; i < c; i += nt) {
    double g = G[i * c + i];
    dsc[i] = g > 0 ? 1.0 / sqrt(g) : 1.0;
  }
  __syncthreads();
  for (int i = tid; i < c * c; i += nt) {
    R[i] = G[i] * dsc[i / c] * dsc[i % c];
    Ri[i] = 0.0;
  }
  __syncthreads();
  __shared__ double maxd;
  __shared__ int bad;
  if (tid == 0) {
    maxd = 0;
    bad = 0;
    for (int i = 0; i < c; ++i) maxd = fmax(maxd, fabs(R[i * c + i]));
  }
  __syncthreads();
  // right-looking Cholesky on the upper triangle: R[k][k..] row k of R
  for (int k = 0; k < c; ++k) {
    if (tid == 0) {
      double d = R[k * c + k];
      if (!(d > 1e-13 * maxd) || !(maxd > 0)) {
        bad = 1;
        d = fmax(fabs(d), 1e-300);
      }
      R[k * c + k] = sqrt(d);
    }
    __syncthreads();
    double rkk = R[k * c + k];
    for (int j = k + 1 + tid; j < c; j += nt) R[k * c + j] /= rkk;
    __syncthreads();
    for (int idx = tid; idx < c * c; idx += nt) {
      int i = idx / c, j = idx % c;
      if (i > k && j >= i) R[i * c + j] -= R[k * c + i] * R[k * c + j];
    }
    __syncthreads();
  }
  // inverse of upper-triangular R: column by column back substitution
  for (int j = tid; j < c; j += nt) {
    for (int i = j; i >= 0; --i) {
      double s = (i == j) ? 1.0 : 0.0;
      for (int k = i + 1; k <= j; ++k) s -= R[i * c + k] * Ri[k * c + j];
      Ri[i * c + j] = s / R[i * c + i];
    }
  }
  __syncthreads();
  for (int i = tid; i < c * c; i += nt) Rinv[i] = Ri[i] * dsc[i / c];
  if (tid == 0) status[0] = bad;
}

// ---------------------------------------------------- Householder (1 CTA)

// deterministic block reduction (warp shuffles, fixed tree); red >= 33 doubles
__device__ double block_sum(double v, double *red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (warp == 0) {
    double w = lane < nw ? red[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) w += __shfl_down_sync(0xffffffffu, w, o);
    if (lane == 0) red[32] = w;
  }
  __syncthreads();
  double r = red[32];
  __syncthreads();
  return r;
}

// A (rows x c) -> explicit Q as dgeqrf + dorgqr; v vectors kept in A,
// Q built in Qout.  One CTA of 1024 threads; used for rank-deficient inputs.
__global__ void __launch_bounds__(1024) householder_kernel(double *A, int rows, int c, double *tau,
                                                           double *Q) {
  __shared__ double red[1024];
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int j = 0; j < c && j < rows; ++j) {
    double s = 0;
    for (int i = j + 1 + tid; i < rows; i += nt) s += A[(size_t)i * c + j] * A[(size_t)i * c + j];
    double sigma = block_sum(s, red);
    double alpha = A[(size_t)j * c + j];
    double t = 0, beta = alpha;
    if (sigma > 0) {
      beta = -copysign(sqrt(alpha * alpha + sigma), alpha);
      t = (beta - alpha) / beta;
      double scal = 1.0 / (alpha - beta);
      for (int i = j + 1 + tid; i < rows; i += nt) A[(size_t)i * c + j] *= scal;
    }
    __syncthreads();
    if (tid == 0) {
      tau[j] = t;
      A[(size_t)j * c + j] = beta;
    }
    __syncthreads();
    // apply H = I - t v v^T to columns j+1..c-1 (v[j] = 1)
    for (int k = j + 1; k < c; ++k) {
      double w = 0;
      for (int i = j + tid; i < rows; i += nt) {
        double v = (i == j) ? 1.0 : A[(size_t)i * c + j];
        w += v * A[(size_t)i * c + k];
      }
      w = block_sum(w, red);
      for (int i = j + tid; i < rows; i += nt) {
        double v = (i == j) ? 1.0 : A[(size_t)i * c + j];
        A[(size_t)i * c + k] -= t * v * w;
      }
      __syncthreads();
    }
  }
  // Q = H_0 ... H_{c-1} [I; 0]
  for (size_t idx = tid; idx < (size_t)rows * c; idx += nt) {
    size_t i = idx / c, k = idx % c;
    Q[idx] = (i == k) ? 1.0 : 0.0;
  }
  __syncthreads();
  for (int j = min(c, rows) - 1; j >= 0; --j) {
    double t = tau[j];
    for (int k = j; k < c; ++k) {
      double w = 0;
      for (int i = j + tid; i < rows; i += nt) {
        double v = (i == j) ? 1.0 : A[(size_t)i * c + j];
        w += v * Q[(size_t)i * c + k];
      }
      w = block_sum(w, red);
      for (int i = j + tid; i < rows; i += nt) {
        double v = (i == j) ? 1.0 : A[(size_t)i * c + j];
        Q[(size_t)i * c + k] -= t * v * w;
      }
      __syncthreads();
    }
  }
}

// --------------------------------------------------------------- Jacobi

__global__ void __launch_bounds__(1024) jacobi_kernel(const double *S, int n, double *w_out,
                                                      double *V_out) {
  extern __shared__ double sm[];
  const int np = (n + 1) & ~1;
  const int ld = np + 1;     // odd row stride: column sweeps hit distinct banks
  double *A = sm;            // np x ld
  double *V = sm + np * ld;  // np x ld
  __shared__ double cs[2 * 64];
  __shared__ int pr[2 * 64];
  __shared__ int order[128];
  __shared__ double red[1024];
  __shared__ int rotated;
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nwarp = nt >> 5;
  for (int idx = tid; idx < np * np; idx += nt) {
    int i = idx / np, j = idx % np;
    A[i * ld + j] = (i < n && j < n) ? S[i * n + j] : 0.0;
    V[i * ld + j] = (i == j) ? 1.0 : 0.0;
  }
  __syncthreads();
  double fro = 0;
  for (int idx = tid; idx < np * np; idx += nt) {
    const double x = A[(idx / np) * ld + idx % np];
    fro += x * x;
  }
  fro = block_sum(fro, red);
  const int half = np / 2;
  for (int sweep = 0; sweep < 60 && np > 1; ++sweep) {
    double off = 0;
    for (int idx = tid; idx < np * np; idx += nt) {
      int i = idx / np, j = idx % np;
      if (i != j) off += A[i * ld + j] * A[i * ld + j];
    }
    off = block_sum(off, red);
    if (!(off > 1e-30 * fro)) break;
    if (tid == 0) rotated = 0;
    __syncthreads();
    for (int step = 0; step < np - 1; ++step) {
      if (tid < half) {
        int k = tid;
        int a = (k == 0) ? 0 : 1 + (k - 1 + step) % (np - 1);
        int kb = np - 1 - k;
        int b = 1 + (kb - 1 + step) % (np - 1);
        int p = min(a, b), q = max(a, b);
        pr[2 * k] = p;
        pr[2 * k + 1] = q;
        const double apq = A[p * ld + q], app = A[p * ld + p], aqq = A[q * ld + q];
        double c = 1.0, s = 0.0;
        // an element below the rounding level of its diagonal pair (or of
        // the whole matrix) is left alone; a sweep that rotates nothing ends
        // the iteration (rounding noise keeps off() from reaching zero)
        const bool negligible = fabs(apq) <= 1e-17 * sqrt(fabs(app * aqq)) || fabs(apq) <= 1e-18 * sqrt(fro);
        if (!negligible) {
          rotated = 1;
          double tau = (aqq - app) / (2.0 * apq);
          double t = (tau >= 0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
          c = 1.0 / sqrt(1.0 + t * t);
          s = t * c;
        }
        cs[2 * k] = c;
        cs[2 * k + 1] = s;
      }
      __syncthreads();
      // warp w applies rotations w, w+32, ...; its lanes stride the rows or
      // columns (no integer division in the sweep)
      for (int k = warp; k < half; k += nwarp) {  // rows: A <- J^T A
        const int p = pr[2 * k], q = pr[2 * k + 1];
        const double c = cs[2 * k], s = cs[2 * k + 1];
        for (int col = lane; col < np; col += 32) {
          const double a = A[p * ld + col], b = A[q * ld + col];
          A[p * ld + col] = c * a - s * b;
          A[q * ld + col] = s * a + c * b;
        }
      }
      __syncthreads();
      for (int k = warp; k < half; k += nwarp) {  // cols: A <- A J, V <- V J
        const int p = pr[2 * k], q = pr[2 * k + 1];
        const double c = cs[2 * k], s = cs[2 * k + 1];
        for (int row = lane; row < np; row += 32) {
          const double a = A[row * ld + p], b = A[row * ld + q];
          A[row * ld + p] = c * a - s * b;
          A[row * ld + q] = s * a + c * b;
          const double va = V[row * ld + p], vb = V[row * ld + q];
          V[row * ld + p] = c * va - s * vb;
          V[row * ld + q] = s * va + c * vb;
        }
      }
      __syncthreads();
    }
    if (rotated == 0) break;
  }
  // sort eigenvalues descending (only the first n indices are real)
  if (tid == 0) {
    for (int i = 0; i < n; ++i) order[i] = i;
    for (int i = 0; i < n; ++i)
      for (int j = i + 1; j < n; ++j)
        if (A[order[j] * ld + order[j]] > A[order[i] * ld + order[i]]) {
          int t = order[i];
          order[i] = order[j];
          order[j] = t;
        }
  }
  __syncthreads();
  for (int i = tid; i < n; i += nt) w_out[i] = A[order[i] * ld + order[i]];
  for (int idx = tid; idx < n * n; idx += nt) {
    int row = idx / n, k = idx % n;
    V_out[idx] = V[row * ld + order[k]];
  }
}

// ------------------------------------------------------------- misc

__global__ void scale_sym_kernel(double *G, int m, const double *sd) {
  size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (size_t)m * m) return;
  int i = (int)(idx / m), j = (int)(idx % m);
  G[idx] *= sd[i] * sd[j];
}

__global__ void clip_rows_kernel(double *U, int n, int r, double delta) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double s = 0;
  for (int j = 0; j < r; ++j) s += U[(size_t)i * r + j] * U[(size_t)i * r + j];
  s = sqrt(s);
  if (delta < s) {  // src/sparse/spsymtensor.cpp:172-183
    double mul = delta / s;
    for (int j = 0; j < r; ++j) U[(size_t)i * r + j] *= mul;
  }
}

template <typename Ts, typename Td>
__global__ void convert_kernel(const Ts *a, Td *b, size_t n) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = (Td)a[i];
}

__global__ void random_fill_kernel(double *A, size_t n, uint64_t seed) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint64_t z = seed + 0x9E3779B97F4A7C15ull * (i + 1);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  A[i] = ((double)(z >> 11) * (1.0 / 9007199254740992.0)) - 0.5;
}

__global__ void eye_kernel(double *I, int s) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < s) I[(size_t)i * s + i] = 1.0;
}

__global__ void copy_cols_kernel(const double *src, int lds, int rows, int cols, double *dst,
                                 int ldd) {
  size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (size_t)rows * cols) return;
  int i = (int)(idx / cols), j = (int)(idx % cols);
  dst[(size_t)i * ldd + j] = src[(size_t)i * lds + j];
}

// residual norms ||S x_i - lam_i x_i|| for i < r
__global__ void residual_kernel(const double *SX, const double *X, int s, int ld, int r,
                                const double *lam, double *res) {
  __shared__ double red[256];
  int i = blockIdx.x;
  double acc = 0;
  for (int row = threadIdx.x; row < s; row += blockDim.x) {
    double d = SX[(size_t)row * ld + i] - lam[i] * X[(size_t)row * ld + i];
    acc += d * d;
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int st = 128; st > 0; st >>= 1) {
    if (threadIdx.x < st) red[threadIdx.x] += red[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) res[i] = sqrt(red[0]);
}

cudaMemPool_t scratch_pool() { return device_pool(); }

struct Scratch {
  void *p = nullptr;
  cudaStream_t st = 0;
  Scratch(size_t bytes, cudaStream_t s) : st(s) {
    if (bytes) SPB_CUDA(cudaMallocFromPoolAsync(&p, bytes, scratch_pool(), st));
  }
  ~Scratch() {
    if (p) cudaFreeAsync(p, st);
  }
  template <class T> T *as() { return reinterpret_cast<T *>(p); }
};

// Partial core products P[chunk][q][j] = sum_{i in chunk} U[i][q0 + q] Y[i][j]
// over FP32 Y (n x m, read once, coalesced along j) and FP64 U (n x r): one
// thread per column j, kCoreRB FP64 accumulators, the U rows of the chunk
// staged in shared memory 64 at a time (every thread reads the same entry).
constexpr int kCoreRB = 16, kCoreRows = 64;
template <typename TY>
__global__ void __launch_bounds__(128) core_partial_kernel(const double *__restrict__ U,
                                                           const TY *__restrict__ Y, int n, int m,
                                                           int r, int q0, int rows_per_chunk,
                                                           double *__restrict__ P) {
  __shared__ double Us[kCoreRows][kCoreRB];
  const int col = blockIdx.x * 128 + threadIdx.x;
  const int i0 = blockIdx.y * rows_per_chunk, i1 = min(n, i0 + rows_per_chunk);
  double acc[kCoreRB];
#pragma unroll
  for (int q = 0; q < kCoreRB; ++q) acc[q] = 0.0;
  for (int ib = i0; ib < i1; ib += kCoreRows) {
    for (int t = threadIdx.x; t < kCoreRows * kCoreRB; t += 128) {
      const int ii = t / kCoreRB, q = t % kCoreRB;
      Us[ii][q] = (ib + ii < i1 && q0 + q < r) ? U[(size_t)(ib + ii) * r + q0 + q] : 0.0;
    }
    __syncthreads();
    const int cnt = min(kCoreRows, i1 - ib);
    if (col < m) {
      for (int ii = 0; ii < cnt; ++ii) {
        const double y = (double)Y[(size_t)(ib + ii) * m + col];
#pragma unroll
        for (int q = 0; q < kCoreRB; ++q) acc[q] = fma(Us[ii][q], y, acc[q]);
      }
    }
    __syncthreads();
  }
  if (col < m) {
#pragma unroll
    for (int q = 0; q < kCoreRB; ++q) P[((size_t)blockIdx.y * kCoreRB + q) * m + col] = acc[q];
  }
}

// core[q0 + q][j] = sum over chunks (in chunk order) of P[chunk][q][j]
__global__ void core_reduce_kernel(const double *__restrict__ P, int chunks, int m, int r, int q0,
                                   double *__restrict__ core) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (size_t)kCoreRB * m) return;
  const int q = (int)(idx / m), j = (int)(idx % m);
  if (q0 + q >= r) return;
  double s = 0.0;
  for (int c = 0; c < chunks; ++c) s += P[((size_t)c * kCoreRB + q) * m + j];
  core[(size_t)(q0 + q) * m + j] = s;
}

}  // namespace

// ------------------------------------------------------------ public API

// C = A^T A (upper tiles computed, the rest mirrored) for a row-major
// K x M matrix A; M even, lda even, A 16-byte aligned.
static void gram_f64(cudaStream_t st, int M, int K, const double *A, int lda, double *C, int ldc) {
  static int nsm = 0;
  if (!nsm) {
    int dev = 0;
    SPB_CUDA(cudaGetDevice(&dev));
    SPB_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  }
  const int nt = (M + GB - 1) / GB;
  const long long tiles = (long long)nt * (nt + 1) / 2;
  // the fewest K splits (each at least 1024 rows) that fill 90% of the
  // waves of one CTA per SM
  int splits = 1;
  for (int s = 1; s <= 8; ++s) {
    if (s > 1 && K / s < 1024) break;
    const long long ctas = tiles * s, waves = (ctas + nsm - 1) / nsm;
    splits = s;
    if ((double)ctas >= 0.9 * (double)(waves * nsm)) break;
  }
  const int kchunk = (int)(cdiv(cdiv(K, splits), GK) * GK);
  splits = std::max(1, (int)cdiv(K, kchunk));
  Scratch ws(sizeof(double) * (size_t)splits * M * M, st);
  const size_t smem = sizeof(GramSmem);
  SPB_CUDA(cudaFuncSetAttribute(gram_tn_f64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  gram_tn_f64_kernel<<<dim3((unsigned)tiles, (unsigned)splits), 256, smem, st>>>(M, K, A, lda, nt, kchunk,
                                                                                 ws.as<double>(), (size_t)M * M);
  SPB_LAUNCH_CHECK();
  gemm_finalize_kernel<double><<<cdiv((long long)M * M, 256), 256, 0, st>>>(M, M, ws.as<double>(), splits,
                                                                           (size_t)M * M, 1.0, 0.0, C, ldc, 1);
  SPB_LAUNCH_CHECK();
}

template <typename T>
void gemm(cudaStream_t st, int M, int N, int K, T alpha, const T *A, int lda, bool transA,
          const T *B, int ldb, bool transB, T beta, T *C, int ldc, const T *kscale,
          bool sym_upper) {
  if (M <= 0 || N <= 0) return;
  if (K <= 0) {
    if (beta == T(0)) {
      for (int i = 0; i < M; ++i) SPB_CUDA(cudaMemsetAsync(C + (size_t)i * ldc, 0, N * sizeof(T), st));
      return;
    }
  }
  if constexpr (std::is_same<T, double>::value) {
    if (!transA && !sym_upper && N <= 16 && M >= 4 * PR && alpha == 1.0 && beta == 0.0) {
      panel_f64_kernel<<<cdiv(M, PR), 256, 0, st>>>(M, N, K, A, lda, B, ldb, transB, kscale, C, ldc);
      SPB_LAUNCH_CHECK();
      return;
    }
    if (transA && !transB && sym_upper && A == B && lda == ldb && M == N && !kscale && M >= GB && M % 2 == 0 &&
        lda % 2 == 0 && (reinterpret_cast<uintptr_t>(A) & 15) == 0 && alpha == 1.0 && beta == 0.0) {
      gram_f64(st, M, K, A, lda, C, ldc);
      return;
    }
  }
  const int tm = cdiv(M, BM), tn = cdiv(N, BN);
  long long tiles = sym_upper ? (long long)tm * (tm + 1) / 2 : (long long)tm * tn;
  int splits = (int)std::max<long long>(1, std::min<long long>((296 + tiles - 1) / tiles, cdiv(K, 256)));
  int kchunk = (int)(cdiv(cdiv(K, splits), BK) * BK);
  splits = std::max(1, (int)cdiv(K, kchunk));
  const bool direct = splits == 1 && alpha == T(1) && beta == T(0) && !sym_upper;
  Scratch ws(direct ? 0 : (size_t)splits * M * N * sizeof(T), st);
  T *out = direct ? C : ws.as<T>();
  const int ldo = direct ? ldc : N;
  const size_t stride = (size_t)M * N;
  dim3 grid(tn, tm, splits);
#define SPB_GEMM_LAUNCH(TA, TB, KS)                                                            \
  gemm_tile_kernel<T, TA, TB, KS><<<grid, 256, 0, st>>>(M, N, K, A, lda, B, ldb, kscale, out, \
                                                        ldo, kchunk, sym_upper ? 1 : 0, stride)
  const bool ks = kscale != nullptr;
  if (transA && transB) { if (ks) SPB_GEMM_LAUNCH(true, true, true); else SPB_GEMM_LAUNCH(true, true, false); }
  else if (transA) { if (ks) SPB_GEMM_LAUNCH(true, false, true); else SPB_GEMM_LAUNCH(true, false, false); }
  else if (transB) { if (ks) SPB_GEMM_LAUNCH(false, true, true); else SPB_GEMM_LAUNCH(false, true, false); }
  else { if (ks) SPB_GEMM_LAUNCH(false, false, true); else SPB_GEMM_LAUNCH(false, false, false); }
#undef SPB_GEMM_LAUNCH
  SPB_LAUNCH_CHECK();
  if (!direct) {
    gemm_finalize_kernel<T><<<cdiv((long long)M * N, 256), 256, 0, st>>>(
        M, N, out, splits, stride, alpha, beta, C, ldc, sym_upper ? 1 : 0);
    SPB_LAUNCH_CHECK();
  }
}

template void gemm<double>(cudaStream_t, int, int, int, double, const double *, int, bool,
                           const double *, int, bool, double, double *, int, const double *, bool);
template void gemm<float>(cudaStream_t, int, int, int, float, const float *, int, bool,
                          const float *, int, bool, float, float *, int, const float *, bool);

template <typename TY>
static void core_from(cudaStream_t st, const double *U, const TY *Y, int n, int m, int r, double *core) {
  if (r <= 0 || m <= 0) return;
  if (n <= 0) {
    SPB_CUDA(cudaMemsetAsync(core, 0, sizeof(double) * (size_t)r * m, st));
    return;
  }
  const int colblocks = (int)cdiv(m, 128);
  // about 8 CTAs per SM in all, each chunk a multiple of the staging depth
  int chunks = std::max(1, std::min((int)cdiv(1184, colblocks), (int)cdiv(n, 4 * kCoreRows)));
  const int rows_per_chunk = (int)(cdiv(cdiv(n, chunks), kCoreRows) * kCoreRows);
  chunks = (int)cdiv(n, rows_per_chunk);
  Scratch part(sizeof(double) * (size_t)chunks * kCoreRB * m, st);
  for (int q0 = 0; q0 < r; q0 += kCoreRB) {
    core_partial_kernel<TY><<<dim3(colblocks, chunks), 128, 0, st>>>(U, Y, n, m, r, q0, rows_per_chunk,
                                                                     part.as<double>());
    SPB_LAUNCH_CHECK();
    core_reduce_kernel<<<cdiv((long long)kCoreRB * m, 256), 256, 0, st>>>(part.as<double>(), chunks, m, r, q0,
                                                                          core);
    SPB_LAUNCH_CHECK();
  }
}

void core_from_f32(cudaStream_t st, const double *U, const float *Y, int n, int m, int r, double *core) {
  core_from<float>(st, U, Y, n, m, r, core);
}
void core_from_f64(cudaStream_t st, const double *U, const double *Y, int n, int m, int r, double *core) {
  core_from<double>(st, U, Y, n, m, r, core);
}

template <typename T>
void weighted_sq(cudaStream_t st, const T *X, const T *Y, const double *w, int rows, int cols,
                 double *d_out2) {
  Scratch part(sizeof(double) * 2 * kRedBlocks, st);
  wsq_partial_kernel<T><<<kRedBlocks, 256, 0, st>>>(X, Y, w, rows, cols, part.as<double>());
  SPB_LAUNCH_CHECK();
  sum_pairs_kernel<<<1, 256, 0, st>>>(part.as<double>(), kRedBlocks, d_out2);
  SPB_LAUNCH_CHECK();
}
template void weighted_sq<double>(cudaStream_t, const double *, const double *, const double *,
                                  int, int, double *);
template void weighted_sq<float>(cudaStream_t, const float *, const float *, const double *, int,
                                 int, double *);

void householder_q(cudaStream_t st, double *A, int rows, int cols) {
  Scratch tau(sizeof(double) * cols, st), Q(sizeof(double) * (size_t)rows * cols, st);
  householder_kernel<<<1, 1024, 0, st>>>(A, rows, cols, tau.as<double>(), Q.as<double>());
  SPB_LAUNCH_CHECK();
  SPB_CUDA(cudaMemcpyAsync(A, Q.p, sizeof(double) * (size_t)rows * cols, cudaMemcpyDeviceToDevice, st));
}

// CholQR2 calls that fell back to Householder QR (reported by the trace)
static int g_householder_fallbacks = 0;

bool orthonormalize(cudaStream_t st, double *A, int rows, int cols) {
  if (cols > 64 || rows < cols) {
    householder_q(st, A, rows, cols);
    return true;
  }
  Scratch G(sizeof(double) * cols * cols, st), Ri(sizeof(double) * cols * cols, st),
      tmp(sizeof(double) * (size_t)rows * cols, st), stat(sizeof(int) * 2, st),
      orig(sizeof(double) * (size_t)rows * cols, st);
  SPB_CUDA(cudaMemcpyAsync(orig.p, A, sizeof(double) * (size_t)rows * cols, cudaMemcpyDeviceToDevice, st));
  int hstat[2] = {0, 0};
  for (int pass = 0; pass < 2; ++pass) {
    gemm<double>(st, cols, cols, rows, 1.0, A, cols, true, A, cols, false, 0.0, G.as<double>(), cols,
                 nullptr, true);
    chol_inv_kernel<<<1, 256, 2 * sizeof(double) * cols * cols, st>>>(G.as<double>(), cols,
                                                                     Ri.as<double>(),
                                                                     stat.as<int>() + pass);
    SPB_LAUNCH_CHECK();
    gemm<double>(st, rows, cols, cols, 1.0, A, cols, false, Ri.as<double>(), cols, false, 0.0,
                 tmp.as<double>(), cols);
    SPB_CUDA(cudaMemcpyAsync(A, tmp.p, sizeof(double) * (size_t)rows * cols,
                             cudaMemcpyDeviceToDevice, st));
  }
  SPB_CUDA(cudaMemcpyAsync(hstat, stat.p, sizeof(int) * 2, cudaMemcpyDeviceToHost, st));
  SPB_CUDA(cudaStreamSynchronize(st));
  if (hstat[0] || hstat[1]) {
    ++g_householder_fallbacks;
    // Gram matrix numerically singular: restart from the original columns
    // with Householder QR, which is stable for any conditioning.
    SPB_CUDA(cudaMemcpyAsync(A, orig.p, sizeof(double) * (size_t)rows * cols, cudaMemcpyDeviceToDevice, st));
    householder_q(st, A, rows, cols);
    return true;
  }
  return false;
}

// W -= Q (Q^T W) twice (classical Gram-Schmidt with re-orthogonalisation)
static void project_out(cudaStream_t st, const double *Q, int ldq, int width, double *W, int s, int b,
                        double *C) {
  if (width <= 0) return;
  for (int pass = 0; pass < 2; ++pass) {
    gemm<double>(st, width, b, s, 1.0, Q, ldq, true, W, b, false, 0.0, C, b);
    gemm<double>(st, s, b, width, -1.0, Q, ldq, false, C, b, false, 1.0, W, b);
  }
}

void jacobi_eig(cudaStream_t st, const double *S, int n, double *w, double *V) {
  if (n > kJacobiMax) fail(SYMPROP_ERR_SIZE, "jacobi_eig: n=%d > %d", n, kJacobiMax);
  int np = (n + 1) & ~1;
  size_t smem = 2 * sizeof(double) * np * (np + 1);
  SPB_CUDA(cudaFuncSetAttribute(jacobi_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  jacobi_kernel<<<1, 1024, smem, st>>>(S, n, w, V);
  SPB_LAUNCH_CHECK();
}

void scale_sym(cudaStream_t st, double *G, int m, const double *sd) {
  scale_sym_kernel<<<cdiv((long long)m * m, 256), 256, 0, st>>>(G, m, sd);
  SPB_LAUNCH_CHECK();
}

void scale_rows_clip(cudaStream_t st, double *U, int n, int r, double delta) {
  clip_rows_kernel<<<cdiv(n, 256), 256, 0, st>>>(U, n, r, delta);
  SPB_LAUNCH_CHECK();
}

template <typename Ts, typename Td> void convert(cudaStream_t st, const Ts *src, Td *dst, size_t n) {
  if (!n) return;
  convert_kernel<Ts, Td><<<cdiv((long long)n, 256), 256, 0, st>>>(src, dst, n);
  SPB_LAUNCH_CHECK();
}
template void convert<double, float>(cudaStream_t, const double *, float *, size_t);
template void convert<float, double>(cudaStream_t, const float *, double *, size_t);

// SPB_TRACE_EIG=1 prints the restart count and final residual of each solve
static bool eig_trace() {
  static const bool on = [] {
    const char *e = std::getenv("SPB_TRACE_EIG");
    return e && *e && *e != '0';
  }();
  return on;
}

// Block Krylov (block Lanczos with full re-orthogonalisation and thick
// restart) for the top-r eigenpairs of S.  Projected problems of at most
// kJacobiMax columns are solved by jacobi_eig.
static int top_eigs_op(cudaStream_t st, const SymApply &apply, int s, int r, double *V, double *lam,
                       const double *warm, double tol, int max_restarts, const double *dense);

int top_eigs(cudaStream_t st, const double *S, int s, int r, double *V, double *lam,
             const double *warm, double tol, int max_restarts) {
  SymApply apply = [S, s](cudaStream_t stream, const double *X, int ldx, int cols, double *Y, int ldy) {
    gemm<double>(stream, s, cols, s, 1.0, S, s, false, X, ldx, false, 0.0, Y, ldy);
  };
  return top_eigs_op(st, apply, s, r, V, lam, warm, tol, max_restarts, S);
}

int top_eigs_op(cudaStream_t st, const SymApply &apply, int s, int r, double *V, double *lam,
                const double *warm, double tol, int max_restarts) {
  return top_eigs_op(st, apply, s, r, V, lam, warm, tol, max_restarts, nullptr);
}

// dense: the matrix itself when it is at hand (small s goes straight to Jacobi)
static int top_eigs_op(cudaStream_t st, const SymApply &apply, int s, int r, double *V, double *lam,
                const double *warm, double tol, int max_restarts, const double *dense) {
  if (r > s) fail(SYMPROP_ERR_INVALID, "rank %d exceeds matrix size %d", r, s);
  if (s <= kJacobiMax) {
    Scratch w(sizeof(double) * s, st), Z(sizeof(double) * s * s, st), Sd(dense ? 0 : sizeof(double) * s * s, st);
    if (!dense) {  // form the small matrix: S = S I
      Scratch I(sizeof(double) * s * s, st);
      SPB_CUDA(cudaMemsetAsync(I.p, 0, sizeof(double) * s * s, st));
      eye_kernel<<<cdiv(s, 256), 256, 0, st>>>(I.as<double>(), s);
      SPB_LAUNCH_CHECK();
      apply(st, I.as<double>(), s, s, Sd.as<double>(), s);
      dense = Sd.as<double>();
    }
    jacobi_eig(st, dense, s, w.as<double>(), Z.as<double>());
    copy_cols_kernel<<<cdiv((long long)s * r, 256), 256, 0, st>>>(Z.as<double>(), s, s, r, V, r);
    SPB_LAUNCH_CHECK();
    SPB_CUDA(cudaMemcpyAsync(lam, w.p, sizeof(double) * r, cudaMemcpyDeviceToHost, st));
    SPB_CUDA(cudaStreamSynchronize(st));
    return SYMPROP_OK;
  }
  const int b = std::min(std::max(r + 8, 2 * r), std::min(48, s));
  if (b < r) fail(SYMPROP_ERR_SIZE, "rank %d too large for the eigensolver", r);
  // Krylov basis width: the Rayleigh-Ritz Jacobi costs O(nb^3) per restart
  // whatever s is, the products with S O(s^2 nb): small matrices take 64
  // columns, large ones the full 96 (fewer restarts); at least two blocks
  const int krylov_cols = s < 1024 ? 64 : kJacobiMax;
  const int nblk = std::max(2, krylov_cols / b);
  const int nb = nblk * b;  // Krylov basis width
  Scratch Q(sizeof(double) * (size_t)s * nb, st), SQ(sizeof(double) * (size_t)s * nb, st),
      T(sizeof(double) * nb * nb, st), w(sizeof(double) * nb, st), Z(sizeof(double) * nb * nb, st),
      C(sizeof(double) * nb * b, st), X(sizeof(double) * (size_t)s * b, st),
      SX(sizeof(double) * (size_t)s * b, st), res(sizeof(double) * b, st),
      blk(sizeof(double) * (size_t)s * b, st);
  double *q = Q.as<double>(), *sq = SQ.as<double>();
  // start block: warm subspace padded with pseudo-random columns
  random_fill_kernel<<<cdiv((long long)s * b, 256), 256, 0, st>>>(X.as<double>(), (size_t)s * b,
                                                                   0x5EED5EEDull);
  SPB_LAUNCH_CHECK();
  if (warm) {
    copy_cols_kernel<<<cdiv((long long)s * r, 256), 256, 0, st>>>(warm, r, s, r, X.as<double>(), b);
    SPB_LAUNCH_CHECK();
  }
  std::vector<double> hw(nb), hres(b);
  for (int it = 0; it <= max_restarts; ++it) {
    // Q[:, 0:b] = orth(X)
    copy_cols_kernel<<<cdiv((long long)s * b, 256), 256, 0, st>>>(X.as<double>(), b, s, b,
                                                                  blk.as<double>(), b);
    SPB_LAUNCH_CHECK();
    orthonormalize(st, blk.as<double>(), s, b);
    copy_cols_kernel<<<cdiv((long long)s * b, 256), 256, 0, st>>>(blk.as<double>(), b, s, b, q, nb);
    SPB_LAUNCH_CHECK();
    int width = b;
    for (int j = 1; j < nblk; ++j) {
      // W = S * Q[:, (j-1)b : jb], orthogonalised against the basis so far
      // (column-scaled CholQR2; Householder when W is numerically rank
      // deficient, then a second projection removes any direction it
      // invented inside the existing basis).
      apply(st, q + (j - 1) * b, nb, b, blk.as<double>(), b);
      project_out(st, q, nb, width, blk.as<double>(), s, b, C.as<double>());
      if (orthonormalize(st, blk.as<double>(), s, b)) {
        project_out(st, q, nb, width, blk.as<double>(), s, b, C.as<double>());
        householder_q(st, blk.as<double>(), s, b);
      }
      copy_cols_kernel<<<cdiv((long long)s * b, 256), 256, 0, st>>>(blk.as<double>(), b, s, b,
                                                                    q + j * b, nb);
      SPB_LAUNCH_CHECK();
      width += b;
    }
    // Rayleigh-Ritz: T = Q^T S Q
    apply(st, q, nb, nb, sq, nb);
    gemm<double>(st, nb, nb, s, 1.0, q, nb, true, sq, nb, false, 0.0, T.as<double>(), nb);
    jacobi_eig(st, T.as<double>(), nb, w.as<double>(), Z.as<double>());
    // X = Q Z[:, :b], SX = SQ Z[:, :b]
    copy_cols_kernel<<<cdiv((long long)nb * b, 256), 256, 0, st>>>(Z.as<double>(), nb, nb, b,
                                                                   C.as<double>(), b);
    SPB_LAUNCH_CHECK();
    gemm<double>(st, s, b, nb, 1.0, q, nb, false, C.as<double>(), b, false, 0.0, X.as<double>(), b);
    gemm<double>(st, s, b, nb, 1.0, sq, nb, false, C.as<double>(), b, false, 0.0, SX.as<double>(), b);
    residual_kernel<<<r, 256, 0, st>>>(SX.as<double>(), X.as<double>(), s, b, r, w.as<double>(),
                                       res.as<double>());
    SPB_LAUNCH_CHECK();
    SPB_CUDA(cudaMemcpyAsync(hw.data(), w.p, sizeof(double) * nb, cudaMemcpyDeviceToHost, st));
    SPB_CUDA(cudaMemcpyAsync(hres.data(), res.p, sizeof(double) * r, cudaMemcpyDeviceToHost, st));
    SPB_CUDA(cudaStreamSynchronize(st));
    double scale = std::max(std::fabs(hw[0]), 1e-300);
    double worst = 0;
    for (int i = 0; i < r; ++i) worst = std::max(worst, hres[i] / scale);
    if (worst <= tol || it == max_restarts) {
      if (eig_trace())
        std::fprintf(stderr, "top_eigs: s=%d r=%d b=%d restarts=%d residual=%.3e tol=%.1e householder=%d\n", s, r,
                     b, it, worst, tol, g_householder_fallbacks);
      g_householder_fallbacks = 0;
      copy_cols_kernel<<<cdiv((long long)s * r, 256), 256, 0, st>>>(X.as<double>(), b, s, r, V, r);
      SPB_LAUNCH_CHECK();
      for (int i = 0; i < r; ++i) lam[i] = hw[i];
      SPB_CUDA(cudaStreamSynchronize(st));
      return worst <= tol ? SYMPROP_OK : SYMPROP_ERR_NOCONV;
    }
  }
  return SYMPROP_ERR_NOCONV;
}

}  // namespace dense

// Stream-ordered scratch from a pool private to this library, one per
// device, that keeps its memory between calls (release threshold: never):
// the eigensolver's many small buffers cost no allocation after the first
// iteration.  (The device's default pool releases
// memory at every synchronisation unless its owner raised the threshold.)
// symprop_trim_memory gives the unused part back.
cudaMemPool_t device_pool() {
  static std::mutex mu;
  static std::map<int, cudaMemPool_t> pools;
  int dev = 0;
  SPB_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  auto it = pools.find(dev);
  if (it != pools.end()) return it->second;
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = dev;
  cudaMemPool_t pool;
  SPB_CUDA(cudaMemPoolCreate(&pool, &props));
  uint64_t keep = ~0ull;
  SPB_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
  pools[dev] = pool;
  return pool;
}

}  // namespace spb
