// S3TTMc, the default schedules: one warp per work item while a row's
// 4 x 4 output tiles fit 3 per lane (order 4 / R <= 16, order 5 / R <= 8,
// ...), otherwise a team of the CTA's 4 warps per work item (order 5 /
// R = 16, order 6 / R = 10, ...).
//
// Same mathematics as the reference's level sweep
// (CompressedDTree::kronecker_product_opt5, src/compressed_dtree.cpp:421-518;
// SymOuterProd, include/detail/dense/symtensor.hpp:24-39):
//     Y[i] += c * K(S),  K(S) = sum_k K(S \ s_k) (x) U[s_k].
// The owners (tree leaves) of a work item are streamed one leaf at a time:
//   * the leaf's N-1 U rows (and c * U rows) are staged in shared memory;
//     the rows of the next leaf are loaded while the current one is
//     computed;
//   * levels 2..N-3 of the recursion are built in shared memory
//     (colexicographic order, see s3ttmc_tiled.cu), one element of all
//     C(N-1, d) tensors of a level per thread, the sub-multisets enumerated
//     at compile time;
//   * the last level is never stored: for each of its 4 x 4 output tiles a
//     thread evaluates the N-1 parent tensors K(S \ s_k) at the tile's 4
//     rows from level N-3 and U in registers, then adds the rank-(N-1)
//     product with the c * U rows.
// Warp kernel: no CTA barrier in the owner loop.  Team kernel: the staging
// and the levels are computed once for the 4 warps, in an (N-2)-deep
// pipeline with one barrier per step (two leaves per step up to order 5).
// A work item is a row, or a slice of at most 256 owners of a long row whose
// FP64 partial sums a second kernel adds in a fixed order.  For a fixed
// prefix p the outputs (p, x), x >= last(p), are consecutive in the
// reference's lexicographic packed order, so a tile row is written at a
// precomputed row offset + x (no permutation table).  FP32 tiles run on the
// paired FMA (fma.rn.f32x2) and each thread folds its plain FP32 sums into
// Kahan pairs in shared memory every 16 owners.
#include <algorithm>
#include <utility>

#include "check.cuh"
#include "s3ttmc_warp.cuh"

namespace spb {
namespace {

constexpr int kWarps = 4, kThreads = kWarps * 32, kMaxL = 7, kMaxNTL = 4;
constexpr int kFold = 16;  // FP32: owners summed plainly between Kahan folds
constexpr uint32_t kURow = 0x80000000u;
constexpr uint32_t kPadRow = 0xffffffffu;

struct WDesc {
  uint32_t dst, nterm;
  uint32_t src[kMaxL], k[kMaxL];
};

struct WarpParams {
  const Chunk *chunks;
  uint32_t nchunks;
  const uint32_t *own_S;
  const void *own_c;
  uint32_t sstride;
  const void *U;
  uint32_t R, R4;
  void *Y;
  uint64_t ldy;
  double *partials;
  uint32_t mL;
  const uint32_t *starts;  // (L+1) x (R+1) colex block starts (DP levels)
  const uint8_t *jtab;
  uint32_t jtab_len, jtab_off[kMaxL + 1];
  const WDesc *desc;
  uint32_t ndesc, desc_begin[kMaxL + 1], desc_count[kMaxL + 1];
  uint32_t lvl_off[kMaxL + 1];  // offset of the first level-d tensor in a staging area
  uint32_t m[kMaxL + 1], m4[kMaxL + 1];
  uint32_t mstr[kMaxL + 1];  // element stride between the level-d tensors (FP64 row padding included)
  uint32_t pair_src[kMaxL * kMaxL];  // level N-3 tensor of the positions other than {k,t}
  const int4 *tiles;                 // per tile: (first row r0 inside block j, j, first column x0, 0)
  const uint4 *rowoff;               // per tile: lex offset - j of its 4 rows, or kPadRow
  uint32_t ntiles;
  uint32_t wsz;                      // per-warp staging elements: 2*L*R4 + ksz4
  uint32_t ksz;                      // elements of the level tensors (levels 2..L-2) in a staging area
  uint64_t nown;                     // bounds the checked build tests
  uint32_t nrows, nslots;
};

template <typename T> __device__ __forceinline__ void ld4(const T *p, T (&v)[4]) {
  if constexpr (sizeof(T) == 4) {
    float4 x = *reinterpret_cast<const float4 *>(p);
    v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
  } else {
    double2 x = *reinterpret_cast<const double2 *>(p), y = *reinterpret_cast<const double2 *>(p + 2);
    v[0] = x.x; v[1] = x.y; v[2] = y.x; v[3] = y.y;
  }
}

__host__ __device__ constexpr int pidx(int k, int t, int L) { return k * L + t; }  // k < t

// (d0, d1) += (a0, a1) * (b0, b1) in one paired FP32 FMA (fma.rn.f32x2,
// sm_100): each lane rounds exactly as a scalar fmaf does
template <typename T>
__device__ __forceinline__ void ffma2(T &d0, T &d1, T a0, T a1, T b0, T b1) {
  static_assert(sizeof(T) == 4, "paired FMA is FP32");
  unsigned long long d, a, b;
  asm("mov.b64 %0, {%1, %2};" : "=l"(d) : "f"(d0), "f"(d1));
  asm("mov.b64 %0, {%1, %2};" : "=l"(a) : "f"(a0), "f"(a1));
  asm("mov.b64 %0, {%1, %2};" : "=l"(b) : "f"(b0), "f"(b1));
  asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(d) : "l"(a), "l"(b));
  asm("mov.b64 {%0, %1}, %2;" : "=f"(d0), "=f"(d1) : "l"(d));
}

// CTAs per SM the register budget is sized for (accumulators: NTL x 16
// values per lane).  With up to 3 tiles per thread FP64 takes 3 CTAs (168
// registers) and FP32 4 (128) up to order 5; from order 6 on (L >= 5) the
// parents of the last level need more registers, and one CTA fewer without
// spills beats the spills (order 6, R = 10, 200k tuples: FP64 9.8 against
// 12.6 ms, FP32 7.2 against 7.5; orders 4 and 5 in FP64 are 15% and 7%
// slower with 2 CTAs).
template <typename T, int NTL, int L> __host__ __device__ constexpr int min_blocks() {
  return sizeof(T) == 8 ? (NTL == 1 ? 4 : (NTL <= 3 && L < 5) ? 3 : 2) : ((NTL <= 3 && L < 5) ? 4 : 3);
}

// Team kernel: owners advanced per pipeline step (two halve the barriers;
// order 6 and up keep one so the (order-1) x 2 staging buffers fit)
__host__ __device__ constexpr int team_owners_per_step(int L) { return L <= 4 ? 2 : 1; }

// U values of one owner staged per lane by the warp kernel (the plan checks
// L * R4 <= 32 * kP)
template <int L> __host__ __device__ constexpr int stage_per_lane() { return L <= 2 ? 4 : 2; }

// Shared tables of the levels 2..L-2 recursion (copied once per CTA).
struct SmemTables {
  uint32_t *start;
  uint8_t *jt;
  WDesc *desc;
  unsigned char *rest;  // first byte after the tables (16-byte aligned)
};

template <int L>
__device__ __forceinline__ SmemTables load_tables(const WarpParams &p, unsigned char *smem, int tid, int nthr) {
  SmemTables tb;
  size_t off = 0;
  tb.start = reinterpret_cast<uint32_t *>(smem + off);
  off += (((size_t)(L + 1) * (p.R + 1) * 4) + 15) / 16 * 16;
  tb.jt = smem + off;
  off += ((size_t)p.jtab_len + 15) / 16 * 16;
  tb.desc = reinterpret_cast<WDesc *>(smem + off);
  off += ((size_t)p.ndesc * sizeof(WDesc) + 15) / 16 * 16;
  tb.rest = smem + off;
  if constexpr (L >= 4) {
    for (uint32_t i = tid; i < (uint32_t)(L + 1) * (p.R + 1); i += nthr) tb.start[i] = p.starts[i];
    for (uint32_t i = tid; i < p.jtab_len; i += nthr) tb.jt[i] = p.jtab[i];
    const uint32_t *src = reinterpret_cast<const uint32_t *>(p.desc);
    uint32_t *dst = reinterpret_cast<uint32_t *>(tb.desc);
    const uint32_t words = p.ndesc * (uint32_t)(sizeof(WDesc) / 4);
    for (uint32_t i = tid; i < words; i += nthr) dst[i] = src[i];
  }
  return tb;
}

// Compile-time enumeration of the sub-multisets of the leaf's L positions
// as L-bit masks, in the order the plan lays their tensors out: by
// popcount, then by increasing mask value.
__host__ __device__ constexpr int popc(int x) { return x ? (x & 1) + popc(x >> 1) : 0; }
__host__ __device__ constexpr int mask_at(int L, int d, int i) {  // i-th mask of popcount d
  int found = 0;
  for (int m = 0; m < (1 << L); ++m)
    if (popc(m) == d) {
      if (found == i) return m;
      ++found;
    }
  return 0;
}
__host__ __device__ constexpr int mask_rank(int L, int m) {  // index among masks of its popcount
  int r = 0;
  for (int x = 0; x < m; ++x) r += popc(x) == popc(m) ? 1 : 0;
  return r + 0 * L;
}
__host__ __device__ constexpr int nmasks(int L, int d) {
  int c = 0;
  for (int m = 0; m < (1 << L); ++m) c += popc(m) == d ? 1 : 0;
  return c;
}

// Storage position of row r of a level tensor.  FP64 inserts 2 doubles
// after every 16 rows: the 4-row groups that lanes fetch with two 128-bit
// loads then fall on distinct banks (row groups 128 bytes apart would
// otherwise share them).  FP32 rows are unpadded (16-byte groups are
// conflict-free).  The host sizes the tensors with level_stride().
template <typename T> __device__ __forceinline__ uint32_t prow(uint32_t r) {
  return sizeof(T) == 8 ? r + 2 * (r >> 4) : r;
}

template <int L, int M, int K, int NS, typename T>
__device__ __forceinline__ void dp_term(T &v, const T (&src)[NS], const T (&uj)[L]) {
  if constexpr (((M >> K) & 1) != 0) {
    constexpr int s = mask_rank(L, M & ~(1 << K));
    v += src[s] * uj[K];
  }
}

template <int L, int D, int I, int NS, typename T, int... K>
__device__ __forceinline__ void dp_mask(T *dst, uint32_t stride, uint32_t e, const T (&src)[NS],
                                        const T (&uj)[L], std::integer_sequence<int, K...>) {
  constexpr int M = mask_at(L, D, I);
  T v = T(0);
  (dp_term<L, M, K, NS, T>(v, src, uj), ...);
  dst[(uint32_t)I * stride + prow<T>(e)] = v;
}

template <int L, int D, int NS, typename T, int... I>
__device__ __forceinline__ void dp_masks(T *dst, uint32_t stride, uint32_t e, const T (&src)[NS],
                                         const T (&uj)[L], std::integer_sequence<int, I...>) {
  (dp_mask<L, D, I, NS, T>(dst, stride, e, src, uj, std::make_integer_sequence<int, L>{}), ...);
}

// Level D (2 <= D <= L-2) of the recursion for one owner: every
// sub-multiset tensor of order D, colex order.  Element e = (row r of
// block j) of all C(L, D) tensors at once:
//   K_D(M)[e] = sum_{k in M} K_{D-1}(M \ k)[r] * U[s_k][j],
// with the C(L, D-1) source values and the L values U[s_k][j] loaded once;
// elements strided over nthr threads.
template <int L, int D, typename T>
__device__ __forceinline__ void dp_level(const WarpParams &p, const SmemTables &tb, const T *sU, T *sK,
                                         uint32_t tid, uint32_t nthr) {
  constexpr int NS = nmasks(L, D - 1);
  const uint32_t R4 = p.R4, md = p.m[D];
  const uint8_t *jt = tb.jt + p.jtab_off[D];
  const uint32_t *stt = tb.start + D * (p.R + 1);
  const T *srcK = sK + p.lvl_off[D - 1];
  const uint32_t sstr = p.mstr[D - 1];
  T *dst = sK + p.lvl_off[D];
  for (uint32_t e = tid; e < md; e += nthr) {
    const uint32_t j = jt[e], r = e - stt[j];
    if (!SPB_BOUND(j < p.R && p.lvl_off[D] + (uint32_t)(nmasks(L, D) - 1) * p.mstr[D] + prow<T>(e) < p.ksz &&
                       (D == 2 ? (uint32_t)(NS - 1) * R4 + r < (uint32_t)L * R4
                               : p.lvl_off[D - 1] + (uint32_t)(NS - 1) * sstr + prow<T>(r) < p.ksz),
                   106, e))
      continue;
    T uj[L], src[NS];
#pragma unroll
    for (int k = 0; k < L; ++k) uj[k] = sU[k * R4 + j];
#pragma unroll
    for (int i = 0; i < NS; ++i) src[i] = (D == 2) ? sU[i * R4 + r] : srcK[i * sstr + prow<T>(r)];
    dp_masks<L, D, NS, T>(dst, p.mstr[D], e, src, uj, std::make_integer_sequence<int, nmasks(L, D)>{});
  }
}

// dp_level for a level d known at run time (2 <= d <= L-2)
template <int L, typename T>
__device__ __forceinline__ void dp_level_rt(int d, const WarpParams &p, const SmemTables &tb, const T *sU, T *sK,
                                            uint32_t tid, uint32_t nthr) {
  if constexpr (L >= 4) if (d == 2) dp_level<L, 2, T>(p, tb, sU, sK, tid, nthr);
  if constexpr (L >= 5) if (d == 3) dp_level<L, 3, T>(p, tb, sU, sK, tid, nthr);
  if constexpr (L >= 6) if (d == 4) dp_level<L, 4, T>(p, tb, sU, sK, tid, nthr);
  if constexpr (L >= 7) if (d == 5) dp_level<L, 5, T>(p, tb, sU, sK, tid, nthr);
}

// The last level for one owner on this thread's tiles: the parents
// K(S \ s_k) at rows (r0+q, j) are
//   sum_{t != k} K(S \ {s_k, s_t})[r0+q] * U[s_t][j]
// (level N-3 tensors, or U rows for order 4), then the tile gets
// sum_k A_k[q] * (c U[s_k])[x0 + cc].
template <int L, int NTL, typename T>
__device__ __forceinline__ void tile_step(const WarpParams &p, const T *sU, const T *sW, const T *sK,
                                          const int4 (&tl)[NTL], const bool (&live)[NTL], T (&acc)[NTL][4][4]) {
  const uint32_t R4 = p.R4;
#pragma unroll
  for (int i = 0; i < NTL; ++i) {
    if (!live[i]) continue;
    const uint32_t r0 = (uint32_t)tl[i].x, jt = (uint32_t)tl[i].y, x0 = (uint32_t)tl[i].z;
    if (!SPB_BOUND(x0 + 3 < R4 && jt < p.R, 105, ((uint64_t)x0 << 32) | jt)) continue;
    T w[L][4], uj[L], A[L][4];
#pragma unroll
    for (int k = 0; k < L; ++k) ld4(sW + k * R4 + x0, w[k]);
#pragma unroll
    for (int t = 0; t < L; ++t) uj[t] = sU[t * R4 + jt];
    if constexpr (L == 2) {
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        A[0][q] = q == 0 ? uj[1] : T(0);
        A[1][q] = q == 0 ? uj[0] : T(0);
      }
    } else {
#pragma unroll
      for (int k = 0; k < L; ++k)
#pragma unroll
        for (int q = 0; q < 4; ++q) A[k][q] = T(0);
#pragma unroll
      for (int k = 0; k < L; ++k)
#pragma unroll
        for (int t = k + 1; t < L; ++t) {
          const uint32_t s = p.pair_src[pidx(k, t, L)];
          T kv[4] = {T(0), T(0), T(0), T(0)};
          if constexpr (L == 3) {
            if (SPB_BOUND((s & 0xffu) * R4 + r0 + 3 < (uint32_t)L * R4, 104, r0)) ld4(sU + (s & 0xffu) * R4 + r0, kv);
          } else {
            if (SPB_BOUND(s + prow<T>(r0 + 3) < p.ksz, 104, r0)) ld4(sK + s + prow<T>(r0), kv);
          }
          if constexpr (sizeof(T) == 4) {  // row pairs on the paired FP32 pipe
#pragma unroll
            for (int h = 0; h < 4; h += 2) {
              ffma2(A[k][h], A[k][h + 1], kv[h], kv[h + 1], uj[t], uj[t]);
              ffma2(A[t][h], A[t][h + 1], kv[h], kv[h + 1], uj[k], uj[k]);
            }
          } else {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              A[k][q] += kv[q] * uj[t];
              A[t][q] += kv[q] * uj[k];
            }
          }
        }
    }
    if constexpr (sizeof(T) == 4) {
#pragma unroll
      for (int cc = 0; cc < 4; ++cc)
#pragma unroll
        for (int h = 0; h < 4; h += 2)
#pragma unroll
          for (int k = 0; k < L; ++k)
            ffma2(acc[i][h][cc], acc[i][h + 1][cc], A[k][h], A[k][h + 1], w[k][cc], w[k][cc]);
    } else {
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) {
          T s = acc[i][q][cc];
#pragma unroll
          for (int k = 0; k < L; ++k) s += A[k][q] * w[k][cc];
          acc[i][q][cc] = s;
        }
    }
  }
}

// FP32: fold the plain sums into the thread's Kahan pairs (sum,
// compensation) kept in shared memory at slot e * stride + me.
template <int NTL, typename T>
__device__ __forceinline__ void kahan_fold(float2 *sK2, uint32_t stride, uint32_t me, T (&acc)[NTL][4][4]) {
#pragma unroll
  for (int i = 0; i < NTL; ++i)
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int cc = 0; cc < 4; ++cc) {
        float2 &ks = sK2[((i * 4 + q) * 4 + cc) * stride + me];
        float2 k = ks;
        const float y = (float)acc[i][q][cc] - k.y;
        const float s2 = k.x + y;
        k.y = (s2 - k.x) - y;
        k.x = s2;
        ks = k;
        acc[i][q][cc] = T(0);
      }
}

template <int NTL, typename T>
__device__ __forceinline__ void kahan_result(const float2 *sK2, uint32_t stride, uint32_t me, T (&acc)[NTL][4][4]) {
#pragma unroll
  for (int i = 0; i < NTL; ++i)
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int cc = 0; cc < 4; ++cc) {
        const float2 k = sK2[((i * 4 + q) * 4 + cc) * stride + me];
        acc[i][q][cc] = (T)(k.x - k.y);
      }
}

// Write this thread's tiles: lex index = row offset + column.
template <int NTL, typename T>
__device__ __forceinline__ void write_tiles(const WarpParams &p, const Chunk &ch, const int4 (&tl)[NTL],
                                            const bool (&live)[NTL], const uint32_t (&ids)[NTL],
                                            const T (&acc)[NTL][4][4]) {
  T *Yrow = reinterpret_cast<T *>(p.Y) + (uint64_t)ch.row * p.ldy;
  double *Prow = p.partials + (uint64_t)ch.slot * p.mL;
#pragma unroll
  for (int i = 0; i < NTL; ++i) {
    if (!live[i]) continue;
    const uint4 ro = p.rowoff[ids[i]];
    const uint32_t rof[4] = {ro.x, ro.y, ro.z, ro.w};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      if (rof[q] == kPadRow) continue;
#pragma unroll
      for (int cc = 0; cc < 4; ++cc) {
        const uint32_t x = (uint32_t)tl[i].z + cc;
        if (x >= p.R || x < (uint32_t)tl[i].y) continue;
        const uint32_t qo = rof[q] + x;
        if (!SPB_BOUND(qo < p.mL, 103, qo)) continue;
        if (ch.slot == kDirect) Yrow[qo] = acc[i][q][cc];
        else Prow[qo] = (double)acc[i][q][cc];
      }
    }
  }
}

// Independent warps: one warp per work item, all of the row's tiles in its
// lanes' registers; no barrier in the owner loop.
template <int L, int NTL, typename T>
__global__ void __launch_bounds__(kThreads, (min_blocks<T, NTL, L>())) s3ttmc_warp_kernel(const WarpParams p) {
  constexpr bool kExact = sizeof(T) == 8;
  constexpr int kP = stage_per_lane<L>();
  extern __shared__ __align__(16) unsigned char smem[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t R = p.R, R4 = p.R4, LR4 = (uint32_t)L * R4;

  const SmemTables tb = load_tables<L>(p, smem, tid, kThreads);
  if constexpr (L >= 4) __syncthreads();
  T *sWarp = reinterpret_cast<T *>(tb.rest);  // kWarps x wsz

  const uint32_t item = blockIdx.x * (uint32_t)kWarps + (uint32_t)warp;
  if (item >= p.nchunks) return;
  const Chunk ch = p.chunks[item];
  if (!SPB_BOUND(ch.ob <= ch.oe && ch.oe <= p.nown && ch.row < p.nrows && (ch.slot == kDirect || ch.slot < p.nslots),
                 101, item))
    return;

  // this lane's tiles: 4 consecutive rows r0..r0+3 of block j (all with last
  // index j) times columns x0..x0+3
  int4 tl[NTL];
  bool live[NTL];
  uint32_t ids[NTL];
#pragma unroll
  for (int i = 0; i < NTL; ++i) {
    ids[i] = (uint32_t)lane + 32u * i;
    live[i] = ids[i] < p.ntiles;
    tl[i] = live[i] ? p.tiles[ids[i]] : make_int4(0, 0, 0, 0);
  }

  // FP64: the row's sums.  FP32: plain sums of the last kFold owners,
  // folded into lane-private Kahan pairs in shared memory, so that one
  // register per output is live across the owner loop.
  T acc[NTL][4][4];
#pragma unroll
  for (int i = 0; i < NTL; ++i)
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[i][a][c] = T(0);
  float2 *sK2 = reinterpret_cast<float2 *>(sWarp + (size_t)kWarps * p.wsz) + (size_t)warp * NTL * 16 * 32;
  if constexpr (!kExact) {
#pragma unroll
    for (int e = 0; e < NTL * 16; ++e) sK2[e * 32 + lane] = make_float2(0.f, 0.f);
  }

  const T *U = reinterpret_cast<const T *>(p.U);
  const T *own_c = reinterpret_cast<const T *>(p.own_c);
  T *sU = sWarp + (size_t)warp * p.wsz;
  T *sW = sU + L * R4;
  T *sK = sW + L * R4;
  int pending = 0;
  // the padding rows of the level tensors are read (and discarded) by the
  // last level: keep them finite
  for (uint32_t i = lane; i < p.wsz; i += 32) sU[i] = T(0);
  __syncwarp();

  // Software pipeline over owners: while owner o is computed, the U rows
  // and coefficient of owner o+1 and the ids of owner o+2 are in flight.
  // Lane k < L holds id k of an owner; the staging lanes fetch it by shuffle.
  auto load_ids = [&](uint64_t o) -> uint32_t {
    const uint32_t id = (o < ch.oe && lane < L) ? p.own_S[o * p.sstride + (uint32_t)lane] : 0u;
    return SPB_BOUND(id < p.nrows, 102, id) ? id : 0u;
  };
  auto load_rows = [&](uint32_t idv, T (&u)[kP]) {
#pragma unroll
    for (int e = 0; e < kP; ++e) {
      const uint32_t i = (uint32_t)lane + 32u * e, k = i / R4, x = i - k * R4;
      const uint32_t s = __shfl_sync(0xffffffffu, idv, (int)(k < (uint32_t)L ? k : 0u));
      u[e] = (i < LR4 && x < R) ? U[(uint64_t)s * R + x] : T(0);
    }
  };
  T u_cur[kP], c_cur = T(0);
  uint32_t ids_next = 0;
  if (ch.ob < ch.oe) {
    load_rows(load_ids(ch.ob), u_cur);
    c_cur = own_c[ch.ob];
    ids_next = load_ids(ch.ob + 1);
  }

  for (uint64_t o = ch.ob; o < ch.oe; ++o) {
#pragma unroll
    for (int e = 0; e < kP; ++e) {
      const uint32_t i = (uint32_t)lane + 32u * e;
      if (i < LR4) {
        sU[i] = u_cur[e];
        sW[i] = c_cur * u_cur[e];
      }
    }
    __syncwarp();
    T u_next[kP], c_next = T(0);
    const bool more = o + 1 < ch.oe;  // warp-uniform
    if (more) {
      load_rows(ids_next, u_next);
      c_next = own_c[o + 1];
    } else {
#pragma unroll
      for (int e = 0; e < kP; ++e) u_next[e] = T(0);
    }
    ids_next = load_ids(o + 2);
    if constexpr (L >= 4) {
#pragma unroll 1
      for (int d = 2; d <= L - 2; ++d) {
        dp_level_rt<L, T>(d, p, tb, sU, sK, (uint32_t)lane, 32u);
        __syncwarp();
      }
    }
    tile_step<L, NTL, T>(p, sU, sW, sK, tl, live, acc);
    if constexpr (!kExact) {
      if (++pending == kFold) {
        pending = 0;
        kahan_fold<NTL, T>(sK2, 32u, (uint32_t)lane, acc);
      }
    }
    __syncwarp();
#pragma unroll
    for (int e = 0; e < kP; ++e) u_cur[e] = u_next[e];
    c_cur = c_next;
  }
  if constexpr (!kExact) {
    kahan_fold<NTL, T>(sK2, 32u, (uint32_t)lane, acc);
    kahan_result<NTL, T>(sK2, 32u, (uint32_t)lane, acc);
  }
  write_tiles<NTL, T>(p, ch, tl, live, ids, acc);
}

// Team of the CTA's 4 warps per work item, for rows with more tiles than
// one warp holds: each thread keeps NTL tiles, and the staging and levels
// 2..L-2 of each owner are computed once for the CTA.  Owner s moves
// through an (L-1)-deep pipeline with one barrier per step: staged at
// step s, level d built at step s+d-1, its tiles added at step s+L-2, each
// owner in its own buffer (L-1 buffers).
template <int L, int NTL, typename T>
__global__ void __launch_bounds__(kThreads, (min_blocks<T, NTL, L>())) s3ttmc_team_kernel(const WarpParams p) {
  constexpr bool kExact = sizeof(T) == 8;
  constexpr int kD = L - 1;                // pipeline depth (steps)
  constexpr int kOps = team_owners_per_step(L);  // owners per step (one barrier each)
  constexpr int kNB = kOps * kD;           // staging buffers
  extern __shared__ __align__(16) unsigned char smem[];
  const uint32_t tid = threadIdx.x;
  const uint32_t R = p.R, R4 = p.R4, LR4 = (uint32_t)L * R4;

  const SmemTables tb = load_tables<L>(p, smem, (int)tid, kThreads);
  T *sBuf = reinterpret_cast<T *>(tb.rest);  // kNB x wsz
  float2 *sK2 = reinterpret_cast<float2 *>(sBuf + (size_t)kNB * p.wsz);
  const Chunk ch = p.chunks[blockIdx.x];
  if (!SPB_BOUND(ch.ob <= ch.oe && ch.oe <= p.nown && ch.row < p.nrows && (ch.slot == kDirect || ch.slot < p.nslots),
                 101, blockIdx.x))
    return;  // the whole CTA leaves (the chunk is the CTA's)

  int4 tl[NTL];
  bool live[NTL];
  uint32_t ids[NTL];
#pragma unroll
  for (int i = 0; i < NTL; ++i) {
    ids[i] = tid + (uint32_t)kThreads * i;
    live[i] = ids[i] < p.ntiles;
    tl[i] = live[i] ? p.tiles[ids[i]] : make_int4(0, 0, 0, 0);
  }
  T acc[NTL][4][4];
#pragma unroll
  for (int i = 0; i < NTL; ++i)
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[i][a][c] = T(0);
  if constexpr (!kExact) {
#pragma unroll
    for (int e = 0; e < NTL * 16; ++e) sK2[e * kThreads + tid] = make_float2(0.f, 0.f);
  }
  // the padding rows of the level tensors are read (and discarded) by the
  // last level: keep them finite
  for (uint32_t i = tid; i < (uint32_t)kNB * p.wsz; i += kThreads) sBuf[i] = T(0);
  __syncthreads();

  const T *U = reinterpret_cast<const T *>(p.U);
  const T *own_c = reinterpret_cast<const T *>(p.own_c);
  const uint64_t nown = ch.oe - ch.ob;
  auto buf = [&](uint64_t o) { return sBuf + (size_t)(o % kNB) * p.wsz; };
  // staging thread tid < kOps*L*R4 owns element (k, x) of owner q of every
  // step; the U value and coefficient of its next owner and the ids of the
  // one after are loaded one step ahead
  const bool stager = tid < (uint32_t)kOps * LR4;
  const uint32_t sq = stager ? tid / LR4 : 0u, se = stager ? tid - sq * LR4 : 0u;
  const uint32_t sk = se / R4, sx = se - sk * R4;
  auto load_id = [&](uint64_t o) -> uint32_t {
    const uint32_t id = (stager && o < nown) ? p.own_S[(ch.ob + o) * p.sstride + sk] : 0u;
    return SPB_BOUND(id < p.nrows, 102, id) ? id : 0u;
  };
  T u_n = T(0), c_n = T(0);
  if (stager && sq < nown) {
    const uint32_t id0 = load_id(sq);
    if (sx < R) u_n = U[(uint64_t)id0 * R + sx];
    c_n = own_c[ch.ob + sq];
  }
  uint32_t id_n = load_id(kOps + sq);
  int pending = 0;
  const uint64_t nsteps = (nown + kOps - 1) / kOps;

  for (uint64_t s = 0; s < nsteps + kD - 1; ++s) {
    if (s < nsteps) {  // stage owners s*kOps .. s*kOps+kOps-1
      const uint64_t o = s * kOps + sq;
      if (stager && o < nown) {
        T *b = buf(o);
        b[se] = u_n;
        b[LR4 + se] = c_n * u_n;
      }
      const uint64_t on = o + kOps;
      u_n = T(0);
      if (stager && on < nown) {
        if (sx < R) u_n = U[(uint64_t)id_n * R + sx];
        c_n = own_c[ch.ob + on];
      }
      id_n = load_id(on + kOps);
    }
    if constexpr (L >= 4) {
#pragma unroll 1
      for (int d = 2; d <= L - 2; ++d) {  // level d of the owners staged d-1 steps ago
        if (s < (uint64_t)(d - 1)) continue;
#pragma unroll
        for (int q = 0; q < kOps; ++q) {
          const uint64_t o = (s - (d - 1)) * kOps + q;
          if (o < nown) {
            T *b = buf(o);
            dp_level_rt<L, T>(d, p, tb, b, b + 2 * LR4, tid, kThreads);
          }
        }
      }
    }
    if (s >= (uint64_t)(kD - 1)) {  // tiles of the owners staged kD-1 steps ago
#pragma unroll
      for (int q = 0; q < kOps; ++q) {
        const uint64_t o = (s - (kD - 1)) * kOps + q;
        if (o >= nown) break;
        const T *b = buf(o);
        tile_step<L, NTL, T>(p, b, b + LR4, b + 2 * LR4, tl, live, acc);
        if constexpr (!kExact) {
          if (++pending == kFold) {
            pending = 0;
            kahan_fold<NTL, T>(sK2, (uint32_t)kThreads, tid, acc);
          }
        }
      }
    }
    __syncthreads();
  }
  if constexpr (!kExact) {
    kahan_fold<NTL, T>(sK2, (uint32_t)kThreads, tid, acc);
    kahan_result<NTL, T>(sK2, (uint32_t)kThreads, tid, acc);
  }
  write_tiles<NTL, T>(p, ch, tl, live, ids, acc);
}

}  // namespace

struct WarpPlan {
  bool ok = false;
  uint32_t L = 0, R = 0, R4 = 0, NTL = 0;
  bool team = false;  // team kernel (4 warps per work item) instead of one warp
  uint32_t m[kMaxL + 1] = {}, m4[kMaxL + 1] = {}, mstr[kMaxL + 1] = {};
  DBuf<uint32_t> starts;
  DBuf<uint8_t> jtab;
  uint32_t jtab_len = 0, jtab_off[kMaxL + 1] = {};
  DBuf<WDesc> desc;
  uint32_t ndesc = 0, desc_begin[kMaxL + 1] = {}, desc_count[kMaxL + 1] = {}, lvl_off[kMaxL + 1] = {};
  uint32_t pair_src[kMaxL * kMaxL] = {};
  DBuf<int4> tiles;
  DBuf<uint4> rowoff;
  uint32_t ntiles = 0, ksz4 = 0, wsz = 0;
  size_t smem[2] = {0, 0};
};

std::shared_ptr<WarpPlan> warp_plan(uint32_t N, uint32_t R) {
  auto pl = std::make_shared<WarpPlan>();
  const uint32_t L = N - 1;
  if (L < 2 || L > (uint32_t)kMaxL || R > 64 || R == 0) return pl;
  pl->L = L;
  pl->R = R;
  pl->R4 = (R + 3) / 4 * 4;
  for (uint32_t d = 0; d <= L; ++d) {
    pl->m[d] = (uint32_t)symsize(R, d);
    pl->m4[d] = (pl->m[d] + 3) / 4 * 4;
    // covers prow<double>(m4 - 1); a multiple of 4 elements so that every
    // tensor starts 16-byte aligned for the FP32 float4 and FP64 double2 loads
    pl->mstr[d] = (pl->m4[d] + 2 * ((pl->m4[d] + 15) / 16) + 3) / 4 * 4;
  }
  if (pl->m[L - 1] >= (1u << 24)) return pl;
  std::vector<uint32_t> starts((size_t)(L + 1) * (R + 1), 0);
  for (uint32_t d = 1; d <= L; ++d)
    for (uint32_t j = 0; j <= R; ++j) starts[(size_t)d * (R + 1) + j] = (uint32_t)symsize(j, d);
  // tiles of the last level, aligned to the colex blocks of the prefixes: a
  // tile is rows r0..r0+3 of block j (prefixes of order L-1 whose last id is
  // j, taken in colex order of the rest) times columns x0..x0+3, x0 from
  // the column block holding j
  auto colex = [](const std::vector<uint32_t> &q) {
    uint64_t cx = 0;
    for (size_t i = 0; i < q.size(); ++i) cx += symsize(q[i], i + 1);
    return cx;
  };
  std::vector<uint32_t> lexL(pl->m[L]);
  for_each_sorted(R, (int)L, [&](const std::vector<uint32_t> &q, uint64_t lin) { lexL[colex(q)] = (uint32_t)lin; });
  // row_off[prefix colex rank] = lex index of (prefix, last) - last
  std::vector<uint32_t> row_off(pl->m[L - 1]);
  for_each_sorted(R, (int)(L - 1), [&](const std::vector<uint32_t> &q, uint64_t) {
    std::vector<uint32_t> full = q;
    full.push_back(q.back());
    row_off[colex(q)] = lexL[colex(full)] - q.back();
  });
  const uint32_t *stP = &starts[(size_t)(L - 1) * (R + 1)];
  std::vector<int4> tiles;
  std::vector<uint4> roff;
  for (uint32_t j = 0; j < R; ++j) {
    const uint32_t base = stP[j], cnt = stP[j + 1] - stP[j];
    for (uint32_t r0 = 0; r0 < cnt; r0 += 4) {
      uint32_t o[4];
      for (uint32_t q = 0; q < 4; ++q) o[q] = (r0 + q < cnt) ? row_off[base + r0 + q] : kPadRow;
      for (uint32_t x0 = j / 4 * 4; x0 < pl->R4; x0 += 4) {
        tiles.push_back(make_int4((int)r0, (int)j, (int)x0, 0));
        roff.push_back(make_uint4(o[0], o[1], o[2], o[3]));
      }
    }
  }
  pl->ntiles = (uint32_t)tiles.size();
  // one warp per work item while the tiles fit 3 per lane (independent
  // warps, no barrier); beyond that the CTA's 4 warps form a team with up to
  // 4 tiles per thread
  pl->team = pl->ntiles > 96;
  const uint32_t slots = pl->team ? (uint32_t)kThreads : 32u;
  pl->NTL = (pl->ntiles + slots - 1) / slots;
  if (pl->NTL > (uint32_t)kMaxNTL) return pl;
  // staging: the warp kernel stages stage_per_lane<L>() values per lane,
  // the team kernel one per thread
  if (!pl->team && L * pl->R4 > (L <= 2 ? 128u : 64u)) return pl;
  if (pl->team && (uint32_t)team_owners_per_step((int)L) * L * pl->R4 > (uint32_t)kThreads) return pl;
  // jtab and descriptors for levels 2..L-2
  std::vector<uint8_t> jt;
  for (uint32_t d = 2; d + 2 <= L; ++d) {
    pl->jtab_off[d] = (uint32_t)jt.size();
    for (uint32_t j = 0; j < R; ++j)
      for (uint32_t e = starts[(size_t)d * (R + 1) + j]; e < starts[(size_t)d * (R + 1) + j + 1]; ++e)
        jt.push_back((uint8_t)j);
  }
  pl->jtab_len = (uint32_t)jt.size();
  std::vector<WDesc> desc;
  std::vector<uint32_t> offm(1u << L, 0);
  uint32_t ksz = 0;
  for (uint32_t d = 2; d + 2 <= L; ++d) {
    pl->desc_begin[d] = (uint32_t)desc.size();
    pl->lvl_off[d] = ksz;  // masks of popcount d follow in increasing order (dp_level relies on it)
    for (uint32_t mask = 0; mask < (1u << L); ++mask) {
      if ((uint32_t)__builtin_popcount(mask) != d) continue;
      WDesc ds{};
      ds.dst = ksz;
      offm[mask] = ksz;
      ksz += pl->mstr[d];
      for (uint32_t k = 0; k < L; ++k) {
        if (!(mask & (1u << k))) continue;
        uint32_t src = mask & ~(1u << k);
        ds.src[ds.nterm] = (d - 1 == 1) ? (kURow | (uint32_t)__builtin_ctz(src)) : offm[src];
        ds.k[ds.nterm] = k;
        ds.nterm++;
      }
      desc.push_back(ds);
    }
    pl->desc_count[d] = (uint32_t)desc.size() - pl->desc_begin[d];
  }
  // the kernels enumerate the masks at compile time: the descriptors only
  // fix the offsets above and are not uploaded
  pl->ndesc = 0;
  pl->ksz4 = ksz;
  if (L >= 3) {
    for (uint32_t k = 0; k < L; ++k)
      for (uint32_t t = k + 1; t < L; ++t) {
        uint32_t rest = ((1u << L) - 1) & ~(1u << k) & ~(1u << t);
        pl->pair_src[pidx((int)k, (int)t, (int)L)] =
            (L - 2 == 1) ? (kURow | (uint32_t)__builtin_ctz(rest)) : offm[rest];
      }
  }
  pl->wsz = 2 * L * pl->R4 + pl->ksz4;
  for (int pi = 0; pi < 2; ++pi) {
    const size_t es = pi == 0 ? 8 : 4;
    size_t fixed = (((size_t)(L + 1) * (R + 1) * 4) + 15) / 16 * 16 + ((size_t)pl->jtab_len + 15) / 16 * 16 +
                   ((size_t)pl->ndesc * sizeof(WDesc) + 15) / 16 * 16;
    // warp kernel: one staging area per warp; team kernel: one per
    // pipeline stage (L-1); FP32 adds the Kahan pairs of every thread
    size_t work = (size_t)(pl->team ? (L - 1) * team_owners_per_step((int)L) : kWarps) * pl->wsz * es;
    if (pi == 1) work = (work + 15) / 16 * 16 + (size_t)kThreads * pl->NTL * 16 * sizeof(float) * 2;
    pl->smem[pi] = fixed + work;
    if (pl->smem[pi] > 200 * 1024) return pl;
  }
  pl->starts.alloc(starts.size());
  SPB_CUDA(cudaMemcpy(pl->starts.p, starts.data(), starts.size() * 4, cudaMemcpyHostToDevice));
  pl->jtab.alloc(std::max<size_t>(jt.size(), 1));
  if (!jt.empty()) SPB_CUDA(cudaMemcpy(pl->jtab.p, jt.data(), jt.size(), cudaMemcpyHostToDevice));
  pl->desc.alloc(std::max<size_t>(desc.size(), 1));
  if (!desc.empty())
    SPB_CUDA(cudaMemcpy(pl->desc.p, desc.data(), desc.size() * sizeof(WDesc), cudaMemcpyHostToDevice));
  pl->tiles.alloc(tiles.size());
  SPB_CUDA(cudaMemcpy(pl->tiles.p, tiles.data(), tiles.size() * sizeof(int4), cudaMemcpyHostToDevice));
  pl->rowoff.alloc(roff.size());
  SPB_CUDA(cudaMemcpy(pl->rowoff.p, roff.data(), roff.size() * sizeof(uint4), cudaMemcpyHostToDevice));
  pl->ok = true;
  return pl;
}

bool warp_supported(const WarpPlan &pl) { return pl.ok; }

template <int L, int NTL, typename T>
static void launch_w(bool team, const WarpParams &wp, uint32_t nchunks, size_t smem, cudaStream_t st) {
  auto kern = team ? s3ttmc_team_kernel<L, NTL, T> : s3ttmc_warp_kernel<L, NTL, T>;
  const uint32_t grid = team ? nchunks : (nchunks + kWarps - 1) / kWarps;
  SPB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kern<<<grid, kThreads, smem, st>>>(wp);
  SPB_LAUNCH_CHECK();
}

template <int L, typename T>
static void launch_w_ntl(uint32_t NTL, bool team, const WarpParams &wp, uint32_t nchunks, size_t smem,
                         cudaStream_t st) {
  switch (NTL) {
    case 1: launch_w<L, 1, T>(team, wp, nchunks, smem, st); break;
    case 2: launch_w<L, 2, T>(team, wp, nchunks, smem, st); break;
    case 3: launch_w<L, 3, T>(team, wp, nchunks, smem, st); break;
    default: launch_w<L, 4, T>(team, wp, nchunks, smem, st); break;
  }
}

template <typename T>
static void launch_w_l(uint32_t L, uint32_t NTL, bool team, const WarpParams &wp, uint32_t nchunks, size_t smem,
                       cudaStream_t st) {
  switch (L) {
    case 2: launch_w_ntl<2, T>(NTL, team, wp, nchunks, smem, st); break;
    case 3: launch_w_ntl<3, T>(NTL, team, wp, nchunks, smem, st); break;
    case 4: launch_w_ntl<4, T>(NTL, team, wp, nchunks, smem, st); break;
    case 5: launch_w_ntl<5, T>(NTL, team, wp, nchunks, smem, st); break;
    case 6: launch_w_ntl<6, T>(NTL, team, wp, nchunks, smem, st); break;
    default: launch_w_ntl<7, T>(NTL, team, wp, nchunks, smem, st); break;
  }
}

void warp_launch(const WarpPlan &pl, const TensorState &t, const ItemSet &items, const void *dU, void *dYpacked,
                 int precision, cudaStream_t st) {
  if (!items.nchunks) return;
  const int pi = precision == SYMPROP_FP64 ? 0 : 1;
  WarpParams wp{};
  wp.chunks = items.chunks;
  wp.nchunks = items.nchunks;
  wp.own_S = t.own_S.p;
  wp.own_c = pi == 0 ? (const void *)t.own_c64.p : (const void *)t.own_c32.p;
  wp.sstride = t.sstride;
  wp.U = dU;
  wp.R = pl.R;
  wp.R4 = pl.R4;
  wp.Y = dYpacked;
  wp.ldy = pl.m[pl.L];
  wp.partials = t.partials.p;
  wp.mL = pl.m[pl.L];
  wp.starts = pl.starts.p;
  wp.jtab = pl.jtab.p;
  wp.jtab_len = pl.jtab_len;
  wp.desc = pl.desc.p;
  wp.ndesc = pl.ndesc;
  for (int d = 0; d <= kMaxL; ++d) {
    wp.jtab_off[d] = pl.jtab_off[d];
    wp.desc_begin[d] = pl.desc_begin[d];
    wp.desc_count[d] = pl.desc_count[d];
    wp.lvl_off[d] = pl.lvl_off[d];
    wp.m[d] = pl.m[d];
    wp.m4[d] = pl.m4[d];
    wp.mstr[d] = pl.mstr[d];
  }
  for (int i = 0; i < kMaxL * kMaxL; ++i) wp.pair_src[i] = pl.pair_src[i];
  wp.tiles = pl.tiles.p;
  wp.rowoff = pl.rowoff.p;
  wp.ntiles = pl.ntiles;
  wp.wsz = pl.wsz;
  wp.ksz = pl.ksz4;
  wp.nown = t.nown;
  wp.nrows = t.dim;
  wp.nslots = t.nslots;
  if (pi == 0) launch_w_l<double>(pl.L, pl.NTL, pl.team, wp, items.nchunks, pl.smem[0], st);
  else launch_w_l<float>(pl.L, pl.NTL, pl.team, wp, items.nchunks, pl.smem[1], st);
  spb_check_host(st, pl.team ? "S3TTMc team kernel" : "S3TTMc warp kernel");
}

}  // namespace spb
