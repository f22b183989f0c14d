/*
 * ORACLE — test infrastructure only.  A plain-C restatement of the reference
 * SymProp S3TTMc path, used by tests/, __graft_entry__.smoke() and the
 * bench's cpu_baseline leg as the CHECKER of the CUDA path.  It is never the
 * product and nothing in symprop_b200/ links or calls it.
 *
 * Pinned against the reference itself: tests/test_oracle.py compares every
 * function here with golden vectors produced by the reference's own compiled
 * code (oracle/_ref, tests/golden/make_golden.py) and with the known-answer
 * values of the reference's tests (tests/test_symtensor.cpp:9-58,
 * tests/test_compressed_dtree.cpp:37-65).
 *
 * Restated pieces (reference file:line):
 *   binomial / packed size ........ include/detail/dense/symtensor_base.hpp:12-30
 *   count_freq, multinomial ....... include/detail/dense/symtensor_base.hpp:42-76
 *   packed offset (At) ............ include/detail/dense/symtensor.hpp:83-94
 *   SymOuterProd .................. include/detail/dense/symtensor.hpp:24-39
 *   packed coefficients ........... include/detail/dense/symtensor.hpp:118-126
 *   unpack (ToTensor) ............. include/detail/dense/symtensor.hpp:96-116
 *   DTree insertion order ......... src/dtree.cpp:38-80
 *   CompressedDTree levels/owners . src/compressed_dtree.cpp:13-90
 *   dep_list ...................... src/compressed_dtree.cpp:92-131
 *   S3TTMc (opt5 math) ............ src/compressed_dtree.cpp:421-518,
 *                                   src/sparse/spsymtensor.cpp:30-110
 *   calc_norm ..................... src/sparse/spsymtensor.cpp:114-138
 *   S3TTMc on listed rows ......... the same owners as S3TTMc, other rows skipped
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_MAXL 16

/* ---------------------------------------------------------------- packed */

uint64_t orc_binomial(uint64_t n, uint64_t k) {
  if (k > n) return 0;
  if (2 * k > n) k = n - k;
  if (k == 0) return 1;
  uint64_t r = n;
  for (uint64_t i = 2; i <= k; i++) {
    r *= (n - i + 1);
    r /= i;
  }
  return r;
}

uint64_t orc_symtens_size(uint64_t dim, uint64_t order) {
  return orc_binomial(order + dim - 1, order);
}

static const uint64_t FACT[21] = {1ULL,
                                  1ULL,
                                  2ULL,
                                  6ULL,
                                  24ULL,
                                  120ULL,
                                  720ULL,
                                  5040ULL,
                                  40320ULL,
                                  362880ULL,
                                  3628800ULL,
                                  39916800ULL,
                                  479001600ULL,
                                  6227020800ULL,
                                  87178291200ULL,
                                  1307674368000ULL,
                                  20922789888000ULL,
                                  355687428096000ULL,
                                  6402373705728000ULL,
                                  121645100408832000ULL,
                                  2432902008176640000ULL};

/* multiplicity of a sorted multiset: n! / prod(freq!) */
uint64_t orc_multinomial_sorted(const uint32_t *s, int n) {
  uint64_t denom = 1;
  int run = 1;
  for (int j = 1; j <= n; j++) {
    if (j < n && s[j] == s[j - 1]) {
      run++;
    } else {
      denom *= FACT[run];
      run = 1;
    }
  }
  return FACT[n] / denom;
}

/* packed offset of a sorted index q[0..N-1] in [0,dim) */
uint64_t orc_packed_offset(const uint32_t *q, int N, uint32_t dim) {
  uint64_t off = 0;
  uint32_t start = 0;
  for (int j = 0; j < N; j++) {
    for (uint32_t i = start; i < q[j]; i++)
      off += orc_symtens_size(dim - i, (uint64_t)(N - 1 - j));
    start = q[j];
  }
  return off;
}

/* next sorted (non-decreasing) index in lexicographic order; 0 at the end */
static int next_sorted(uint32_t *q, int N, uint32_t dim) {
  for (int j = N - 1; j >= 0; j--) {
    if (q[j] + 1 < dim) {
      q[j]++;
      for (int k = j + 1; k < N; k++) q[k] = q[j];
      return 1;
    }
  }
  return 0;
}

/* packed enumeration: writes m*N indices (row-major) */
void orc_packed_indices(uint32_t dim, int N, uint32_t *out) {
  uint32_t q[ORC_MAXL] = {0};
  uint64_t p = 0;
  if (dim == 0) return;
  do {
    memcpy(out + p * N, q, sizeof(uint32_t) * N);
    p++;
  } while (next_sorted(q, N, dim));
}

void orc_symtens_coeff(uint32_t dim, int N, double *coeff) {
  uint32_t q[ORC_MAXL] = {0};
  uint64_t p = 0;
  do {
    coeff[p++] = (double)orc_multinomial_sorted(q, N);
  } while (next_sorted(q, N, dim));
}

/* dst (order L) += SymOuterProd(src (order L-1), row) */
void orc_sym_outer_prod(double *restrict dst, const double *restrict src, const double *restrict row,
                        uint32_t dim, int L) {
  if (L == 1) {
    for (uint32_t c = 0; c < dim; c++) dst[c] += src[0] * row[c];
    return;
  }
  uint32_t q[ORC_MAXL] = {0};
  uint64_t in = 0, out = 0;
  do {
    for (uint32_t last = q[L - 2]; last < dim; last++)
      dst[out++] += src[in] * row[last];
    in++;
  } while (next_sorted(q, L - 1, dim));
}

/* unpack packed order-N data into dim^N full tensor */
void orc_unpack(const double *packed, uint32_t dim, int N, double *full) {
  uint64_t total = 1;
  for (int j = 0; j < N; j++) total *= dim;
  uint32_t idx[ORC_MAXL], s[ORC_MAXL];
  for (uint64_t f = 0; f < total; f++) {
    uint64_t x = f;
    for (int j = N - 1; j >= 0; j--) {
      idx[j] = (uint32_t)(x % dim);
      x /= dim;
    }
    memcpy(s, idx, sizeof(uint32_t) * N);
    for (int a = 1; a < N; a++) { /* insertion sort */
      uint32_t v = s[a];
      int b = a - 1;
      while (b >= 0 && s[b] > v) {
        s[b + 1] = s[b];
        b--;
      }
      s[b + 1] = v;
    }
    full[f] = packed[orc_packed_offset(s, N, dim)];
  }
}

/* ------------------------------------------------------------- S3TTMc */

/* K(S) for a sorted multiset S of size L (0-based ids) by the level
 * recursion K(S) = sum_k K(S \ s_k) (x) U[s_k], memoised over position
 * subsets.  out has symtens_size(R, L) entries. */
static void leaf_tensor(const uint32_t *S, int L, const double *U, uint32_t R,
                        double *out) {
  int nmask = 1 << L;
  double **K = (double **)calloc((size_t)nmask, sizeof(double *));
  for (int mask = 1; mask < nmask; mask++) {
    int pc = __builtin_popcount((unsigned)mask);
    uint64_t sz = orc_symtens_size(R, (uint64_t)pc);
    K[mask] = (double *)calloc(sz, sizeof(double));
    if (pc == 1) {
      int k = __builtin_ctz((unsigned)mask);
      memcpy(K[mask], U + (uint64_t)S[k] * R, sizeof(double) * R);
      continue;
    }
    for (int k = 0; k < L; k++) {
      if (!(mask & (1 << k))) continue;
      orc_sym_outer_prod(K[mask], K[mask & ~(1 << k)], U + (uint64_t)S[k] * R,
                         R, pc);
    }
  }
  memcpy(out, K[nmask - 1], sizeof(double) * orc_symtens_size(R, (uint64_t)L));
  for (int mask = 1; mask < nmask; mask++) free(K[mask]);
  free(K);
}

/* Y (dim x ldy, row-major) = S3TTMc of the tensor with U (dim x R).
 * inds: nnz x order sorted 1-based ids.  packed != 0 -> ldy = C(R+N-2, N-1),
 * else ldy = R^(N-1) with rows unpacked. */
int orc_s3ttmc(uint32_t order, uint32_t dim, uint64_t nnz, const uint32_t *inds,
               const double *vals, uint32_t R, const double *U, int packed,
               double *Y) {
  int N = (int)order, L = N - 1;
  if (N < 2 || N > ORC_MAXL) return -1;
  uint64_t m = orc_symtens_size(R, (uint64_t)L);
  uint64_t ldy = m;
  if (!packed) {
    ldy = 1;
    for (int j = 0; j < L; j++) ldy *= R;
  }
  memset(Y, 0, sizeof(double) * ldy * dim);
  double *Kbuf = (double *)malloc(sizeof(double) * m);
  uint32_t t[ORC_MAXL], S[ORC_MAXL];
  for (uint64_t i = 0; i < nnz; i++) {
    for (int j = 0; j < N; j++) t[j] = inds[i * N + j] - 1;
    double coef = vals[i] * (double)orc_multinomial_sorted(t, N) /
                  (double)FACT[N];
    if (N == 2) continue; /* reference: empty level loop, Y stays 0 */
    for (int j = N - 1; j >= 0; j--) {
      int c = 0;
      for (int k = 0; k < N; k++)
        if (k != j) S[c++] = t[k];
      leaf_tensor(S, L, U, R, Kbuf);
      double *y = Y + (uint64_t)t[j] * ldy;
      for (uint64_t q = 0; q < m; q++) y[q] += coef * Kbuf[q];
    }
  }
  free(Kbuf);
  if (!packed) {
    double *row = (double *)malloc(sizeof(double) * m);
    for (uint32_t i = 0; i < dim; i++) {
      memcpy(row, Y + (uint64_t)i * ldy, sizeof(double) * m);
      orc_unpack(row, R, L, Y + (uint64_t)i * ldy);
    }
    free(row);
  }
  return 0;
}

/* K(S) as leaf_tensor computes it, with the level tensors in a caller-owned
 * workspace (one block of orc_leaf_ws_size(R, L) doubles) instead of one
 * allocation per position subset. */
static uint64_t orc_leaf_ws_size(uint32_t R, int L) {
  uint64_t tot = 0;
  for (int mask = 1; mask < (1 << L); mask++)
    tot += orc_symtens_size(R, (uint64_t)__builtin_popcount((unsigned)mask));
  return tot;
}

static void leaf_tensor_ws(const uint32_t *S, int L, const double *U, uint32_t R,
                           double *ws, double *out) {
  double *K[1 << 12]; /* L <= 12 (checked by the caller) */
  double *next = ws;
  for (int mask = 1; mask < (1 << L); mask++) {
    int pc = __builtin_popcount((unsigned)mask);
    uint64_t sz = orc_symtens_size(R, (uint64_t)pc);
    K[mask] = next;
    next += sz;
    if (pc == 1) {
      memcpy(K[mask], U + (uint64_t)S[__builtin_ctz((unsigned)mask)] * R, sizeof(double) * R);
      continue;
    }
    memset(K[mask], 0, sizeof(double) * sz);
    for (int k = 0; k < L; k++) {
      if (!(mask & (1 << k))) continue;
      orc_sym_outer_prod(K[mask], K[mask & ~(1 << k)], U + (uint64_t)S[k] * R, R, pc);
    }
  }
  memcpy(out, K[(1 << L) - 1], sizeof(double) * orc_symtens_size(R, (uint64_t)L));
}

/* The packed Y of orc_s3ttmc restricted to the listed rows: Yrows[k] is
 * row rows[k] (0-based ids, distinct), nrows x C(R+N-2, N-1).  The owners
 * are those of orc_s3ttmc (every tuple, every removed position j, Y[t_j] +=
 * coef K(S)), and the owners of unlisted rows are skipped, so checking a few
 * rows of a large tensor costs only their owners.  The owners are divided
 * among OpenMP threads, each summing into its own copy of the listed rows;
 * the copies are added at the end. */
int orc_s3ttmc_rows(uint32_t order, uint32_t dim, uint64_t nnz, const uint32_t *inds,
                    const double *vals, uint32_t R, const double *U, uint64_t nrows,
                    const uint32_t *rows, double *Yrows) {
  int N = (int)order, L = N - 1;
  if (N < 2 || N > ORC_MAXL || L > 12) return -1;
  uint64_t m = orc_symtens_size(R, (uint64_t)L);
  memset(Yrows, 0, sizeof(double) * m * nrows);
  if (N == 2 || nrows == 0) return 0; /* reference: empty level loop, Y stays 0 */
  int64_t *slot = (int64_t *)malloc(sizeof(int64_t) * dim);
  if (!slot) return -2;
  for (uint32_t i = 0; i < dim; i++) slot[i] = -1;
  for (uint64_t k = 0; k < nrows; k++) {
    if (rows[k] >= dim || slot[rows[k]] >= 0) {
      free(slot);
      return -1;
    }
    slot[rows[k]] = (int64_t)k;
  }
  uint64_t wsz = orc_leaf_ws_size(R, L);
  int fail = 0;
#pragma omp parallel
  {
    double *mine = (double *)calloc(m * nrows, sizeof(double));
    double *ws = (double *)malloc(sizeof(double) * wsz);
    double *Kbuf = (double *)malloc(sizeof(double) * m);
    if (!mine || !ws || !Kbuf) {
#pragma omp atomic write
      fail = 1;
    } else {
      uint32_t t[ORC_MAXL], S[ORC_MAXL];
#pragma omp for schedule(dynamic, 256)
      for (uint64_t i = 0; i < nnz; i++) {
        int any = 0;
        for (int j = 0; j < N; j++) {
          t[j] = inds[i * N + j] - 1;
          any |= slot[t[j]] >= 0;
        }
        if (!any) continue;
        double coef = vals[i] * (double)orc_multinomial_sorted(t, N) / (double)FACT[N];
        for (int j = N - 1; j >= 0; j--) {
          int64_t k = slot[t[j]];
          if (k < 0) continue;
          int c = 0;
          for (int q = 0; q < N; q++)
            if (q != j) S[c++] = t[q];
          leaf_tensor_ws(S, L, U, R, ws, Kbuf);
          double *y = mine + (uint64_t)k * m;
          for (uint64_t q = 0; q < m; q++) y[q] += coef * Kbuf[q];
        }
      }
#pragma omp critical
      for (uint64_t q = 0; q < m * nrows; q++) Yrows[q] += mine[q];
    }
    free(mine);
    free(ws);
    free(Kbuf);
  }
  free(slot);
  return fail ? -2 : 0;
}

double orc_norm(uint32_t order, uint64_t nnz, const uint32_t *inds,
                const double *vals) {
  double s = 0.0;
  for (uint64_t i = 0; i < nnz; i++)
    s += vals[i] * vals[i] *
         (double)orc_multinomial_sorted(inds + i * order, (int)order);
  return sqrt(s);
}

/* --------------------------------------------------------------- tree */

typedef struct {
  int depth;          /* order - 1 */
  uint64_t size[ORC_MAXL];
  uint32_t *keys[ORC_MAXL]; /* size[l] x (l+1) sorted multisets, 1-based */
  uint64_t *ptr[ORC_MAXL];  /* size[l]+1 */
  uint64_t *dep[ORC_MAXL];  /* size[l] x (l+1), l >= 1 */
  uint64_t nown;
  uint64_t *own_rem;
  double *own_val;
} orc_tree;

static int g_cmp_len;
static int cmp_keys(const void *a, const void *b) {
  const uint32_t *x = (const uint32_t *)a, *y = (const uint32_t *)b;
  for (int j = 0; j < g_cmp_len; j++) {
    if (x[j] != y[j]) return x[j] < y[j] ? -1 : 1;
  }
  return 0;
}
/* owners: key (N-1 ids) followed by the insertion sequence number (2 words) */
static int cmp_owner(const void *a, const void *b) {
  int c = cmp_keys(a, b);
  if (c) return c;
  const uint32_t *x = (const uint32_t *)a + g_cmp_len,
                 *y = (const uint32_t *)b + g_cmp_len;
  uint64_t sx = ((uint64_t)x[0] << 32) | x[1], sy = ((uint64_t)y[0] << 32) | y[1];
  return sx < sy ? -1 : (sx > sy);
}

static uint64_t find_key(const uint32_t *keys, uint64_t n, int len,
                         const uint32_t *k) {
  uint64_t lo = 0, hi = n;
  g_cmp_len = len;
  while (lo < hi) {
    uint64_t mid = (lo + hi) / 2;
    if (cmp_keys(keys + mid * len, k) < 0)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

/* Level l holds every sorted (l+1)-sub-multiset of the tuples, in
 * lexicographic order (the BFS order of a trie whose children are sorted by
 * value, src/compressed_dtree.cpp:25-62).  The owners of a leaf are listed
 * in insertion order: nonzero ascending, and for each nonzero the removed
 * position runs N-1 down to 0 (src/dtree.cpp:62-80). */
orc_tree *orc_tree_build(uint32_t order, uint32_t dim, uint64_t nnz,
                         const uint32_t *inds, const double *vals) {
  (void)dim;
  int N = (int)order;
  if (N < 2 || N > ORC_MAXL) return NULL;
  orc_tree *T = (orc_tree *)calloc(1, sizeof(orc_tree));
  T->depth = N - 1;
  for (int l = 0; l < T->depth; l++) {
    int len = l + 1;
    /* all position subsets of size len */
    uint64_t per = orc_binomial((uint64_t)N, (uint64_t)len);
    uint32_t *buf = (uint32_t *)malloc(sizeof(uint32_t) * len * per * (nnz ? nnz : 1));
    uint64_t cnt = 0;
    for (uint64_t i = 0; i < nnz; i++) {
      const uint32_t *t = inds + i * N;
      for (unsigned mask = 0; mask < (1u << N); mask++) {
        if (__builtin_popcount(mask) != len) continue;
        int c = 0;
        for (int k = 0; k < N; k++)
          if (mask & (1u << k)) buf[cnt * len + c++] = t[k];
        cnt++;
      }
    }
    g_cmp_len = len;
    qsort(buf, cnt, sizeof(uint32_t) * len, cmp_keys);
    uint64_t u = 0;
    for (uint64_t i = 0; i < cnt; i++) {
      if (u == 0 || cmp_keys(buf + (u - 1) * len, buf + i * len) != 0) {
        memmove(buf + u * len, buf + i * len, sizeof(uint32_t) * len);
        u++;
      }
    }
    T->size[l] = u;
    T->keys[l] = buf;
  }
  /* child pointers: children of node j at level l are level-(l+1) nodes with
   * prefix keys[l][j] */
  for (int l = 0; l + 1 < T->depth; l++) {
    int len = l + 1;
    T->ptr[l] = (uint64_t *)malloc(sizeof(uint64_t) * (T->size[l] + 1));
    uint64_t c = 0;
    for (uint64_t j = 0; j < T->size[l]; j++) {
      T->ptr[l][j] = c;
      g_cmp_len = len;
      while (c < T->size[l + 1] &&
             cmp_keys(T->keys[l + 1] + c * (len + 1), T->keys[l] + j * len) == 0)
        c++;
    }
    T->ptr[l][T->size[l]] = c;
  }
  /* dep lists */
  for (int l = 1; l < T->depth; l++) {
    int len = l + 1;
    T->dep[l] = (uint64_t *)malloc(sizeof(uint64_t) * T->size[l] * len);
    uint32_t sub[ORC_MAXL];
    for (uint64_t j = 0; j < T->size[l]; j++) {
      const uint32_t *key = T->keys[l] + j * len;
      for (int k = 0; k < len; k++) {
        int c = 0;
        for (int x = 0; x < len; x++)
          if (x != k) sub[c++] = key[x];
        T->dep[l][j * len + k] = find_key(T->keys[l - 1], T->size[l - 1], len - 1, sub);
      }
    }
  }
  /* owners */
  {
    int L = N - 1;
    int w = L + 2;
    uint32_t *ob = (uint32_t *)malloc(sizeof(uint32_t) * w * N * (nnz ? nnz : 1));
    uint64_t o = 0;
    for (uint64_t i = 0; i < nnz; i++) {
      const uint32_t *t = inds + i * N;
      for (int j = N - 1; j >= 0; j--) {
        int c = 0;
        for (int k = 0; k < N; k++)
          if (k != j) ob[o * w + c++] = t[k];
        uint64_t seq = i * (uint64_t)N + (uint64_t)(N - 1 - j);
        ob[o * w + L] = (uint32_t)(seq >> 32);
        ob[o * w + L + 1] = (uint32_t)seq;
        o++;
      }
    }
    g_cmp_len = L;
    qsort(ob, o, sizeof(uint32_t) * w, cmp_owner);
    T->nown = o;
    T->own_rem = (uint64_t *)malloc(sizeof(uint64_t) * (o ? o : 1));
    T->own_val = (double *)malloc(sizeof(double) * (o ? o : 1));
    int lv = T->depth - 1;
    T->ptr[lv] = (uint64_t *)calloc(T->size[lv] + 1, sizeof(uint64_t));
    uint64_t leaf = 0;
    for (uint64_t x = 0; x < o; x++) {
      uint64_t seq = ((uint64_t)ob[x * w + L] << 32) | ob[x * w + L + 1];
      uint64_t i = seq / (uint64_t)N;
      int j = N - 1 - (int)(seq % (uint64_t)N);
      T->own_rem[x] = inds[i * N + j];
      T->own_val[x] = vals[i];
      g_cmp_len = L;
      while (cmp_keys(T->keys[lv] + leaf * L, ob + x * w) != 0) {
        leaf++;
        T->ptr[lv][leaf] = x;
      }
    }
    for (uint64_t lf = leaf + 1; lf <= T->size[lv]; lf++) T->ptr[lv][lf] = o;
    free(ob);
  }
  return T;
}

int orc_tree_depth(const orc_tree *T) { return T->depth; }
uint64_t orc_tree_level_size(const orc_tree *T, int l) { return T->size[l]; }
uint64_t orc_tree_nowners(const orc_tree *T) { return T->nown; }

/* level_idx[l] (last id of each node), level_ptr[l], dep_list[l]; and the
 * full keys (size x (l+1)) */
void orc_tree_copy_level(const orc_tree *T, int l, uint32_t *idx, uint64_t *ptr,
                         uint64_t *dep, uint32_t *keys) {
  int len = l + 1;
  for (uint64_t j = 0; j < T->size[l]; j++) {
    if (idx) idx[j] = T->keys[l][j * len + len - 1];
  }
  if (ptr && T->ptr[l]) memcpy(ptr, T->ptr[l], sizeof(uint64_t) * (T->size[l] + 1));
  if (dep && l >= 1) memcpy(dep, T->dep[l], sizeof(uint64_t) * T->size[l] * len);
  if (keys) memcpy(keys, T->keys[l], sizeof(uint32_t) * T->size[l] * len);
}

void orc_tree_copy_owners(const orc_tree *T, uint64_t *rem, double *val) {
  memcpy(rem, T->own_rem, sizeof(uint64_t) * T->nown);
  memcpy(val, T->own_val, sizeof(double) * T->nown);
}

void orc_tree_free(orc_tree *T) {
  if (!T) return;
  for (int l = 0; l < T->depth; l++) {
    free(T->keys[l]);
    free(T->ptr[l]);
    free(T->dep[l]);
  }
  free(T->own_rem);
  free(T->own_val);
  free(T);
}
