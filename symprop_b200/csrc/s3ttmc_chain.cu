// S3TTMc, pivot-chain schedule (order 4 / R <= 16): the owners of a row are
// contracted pivot by pivot instead of leaf by leaf.
//
// The reference's leaf tensor (SymOuterProd recursion,
// include/detail/dense/symtensor.hpp:24-39, src/compressed_dtree.cpp:421-518)
// is, for a leaf S = {s_1, s_2, s_3} and sorted column indices q,
//     K(S)[q0 q1 q2] = sum over the 6 orderings of S of prod_k U[s_pi(k)][q_k]
//                    = sum_t U[s_1][q_t] * K({s_2, s_3})[q without q_t]
// for any choice of the position s_1, and K({s_2, s_3})[x, y] =
// U[s_2][x] U[s_3][y] + U[s_3][x] U[s_2][y].  With every leaf ordered by node
// degree (s_1 the node of highest degree) and a row's owners sorted by
// (s_1, s_2), the row is
//     Y[i] = Sym3(G),   G = sum_{s_1} U[s_1] (x) Q_{s_1}                (16 x m2)
//     Q_{s_1} = sum_{s_2} U[s_2] (x)s W_{s_1 s_2}                         (m2 = R(R+1)/2)
//     W_{s_1 s_2} = sum over its owners of c * U[s_3]                     (R)
// with Sym3(G)[q0 q1 q2] = G[q0][q1 q2] + G[q1][q0 q2] + G[q2][q0 q1] and
// (x)s the symmetric outer product.  Hub rows share their high-degree
// pivots across many owners: on the order-4 Zipf(1.1) workload a row has
// 0.11 distinct s_1 and 0.50 distinct (s_1, s_2) per owner, so the row
// costs about 16 + 0.50 * 272 + 0.11 * 2176 FMAs per owner, against about
// 3,300 for the leaf-by-leaf schedule.  The sums are the reference's,
// associated differently (FP64 results agree to rounding).
//
// Kernel: one CTA of 128 threads per work item (a row, or a slice of a long
// row whose partial rows the combine kernel adds).  Owners are taken in
// batches of up to 256 with at most kSG (s_1, s_2) subgroups and kG s_1
// groups (49 KB of shared memory in FP64: 4 CTAs per SM); a batch boundary
// (or slice boundary) may cut a group: by linearity the two parts add up.
// Per batch: W of every subgroup (8 lanes over contiguous owner ranges,
// carries between lanes), then Q of every group as 4 x 4 register tiles
// (shared memory), then each thread adds its 18 entries of G.  The row's G
// then goes through shared memory (odd row stride) for Sym3.  FP32: the
// batch's G is summed in FP32 and folded into FP64 totals after every batch.
#include <cub/cub.cuh>

#include <algorithm>
#include <map>
#include <mutex>

#include "check.cuh"
#include "s3ttmc_chain.cuh"

namespace spb {
namespace {

constexpr int kThreads = 128;
constexpr int kB = 256;   // owners per batch
constexpr int kSG = 80;   // (s_1, s_2) subgroups per batch
constexpr int kG = 16;    // s_1 groups per batch
constexpr int kRP = 16;   // R padded
constexpr int kM2 = 136;  // packed order-2 entries at R = 16
constexpr int kS2 = kM2 + 1;  // shared row stride of 16 x kM2 arrays: odd, so rows q, q+1, ... hit different banks
constexpr int kBeta = 9;  // beta slots per thread: 16 x 9 >= kM2

struct ChainParams {
  const Chunk *chunks;
  uint32_t nchunks;
  const uint32_t *S;  // nown x sstride, leaf ids in pivot order
  uint32_t sstride;
  const void *c;      // coefficients (T)
  const uint8_t *flags;
  const void *U;      // n x R (T)
  uint32_t R, m2, m3;
  void *Y;            // packed rows (T), row stride m3
  double *partials;   // nslots x m3
  const uint32_t *trip;  // m3 packed (q0 | q1 << 8 | q2 << 16), lexicographic
  uint64_t nown;
  uint32_t nrows, nslots;
};

__device__ __forceinline__ uint32_t pair_index(uint32_t x, uint32_t y, uint32_t R) {  // x <= y
  return x * R - (x * (x - 1)) / 2 + (y - x);
}

template <typename T> struct Smem {
  uint32_t s1[kB], s2[kB], s3[kB];
  uint8_t px[kM2], py[kM2];  // packed order-2 index -> (x <= y)
  T c[kB];
  uint16_t sg_start[kSG + 1], g_sg[kG + 1];
  uint32_t sg_s2[kSG], g_s1[kG];
  uint8_t sg_of[kB];             // subgroup of each owner of the batch
  T carry[kThreads / 16][kRP];   // W of a subgroup begun in an earlier lane
  int carry_sg[kThreads / 16];
  uint32_t warp_tot[kThreads / 32];
  int nb, nsg, ng;
  union __align__(16) {
    struct {
      T W[kSG][kRP], U2[kSG][kRP];
      T Q[kG][kM2];
      T U1[kG][kRP];
    } b;                        // one batch
    double G[kRP * kS2];        // the row's G at the end (FP64, row stride kS2)
  } u;
};

// Four consecutive values from shared memory (16-byte aligned).
__device__ __forceinline__ void load4(const double *p, double (&v)[4]) {
  const double2 a = reinterpret_cast<const double2 *>(p)[0], b = reinterpret_cast<const double2 *>(p)[1];
  v[0] = a.x, v[1] = a.y, v[2] = b.x, v[3] = b.y;
}
__device__ __forceinline__ void load4(const float *p, float (&v)[4]) {
  const float4 a = *reinterpret_cast<const float4 *>(p);
  v[0] = a.x, v[1] = a.y, v[2] = a.z, v[3] = a.w;
}

// Asynchronous 16-byte copy global -> shared (both 16-byte aligned).
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Pull the 128-byte line holding a row of U into L1 ahead of its gather.
__device__ __forceinline__ void prefetch_l1(const void *p) {
  asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

// Inclusive scan over the CTA of 32-bit values (two 16-bit counts packed).
__device__ __forceinline__ uint32_t cta_scan(uint32_t v, uint32_t *warp_tot) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t u = __shfl_up_sync(0xffffffffu, v, d);
    if (lane >= d) v += u;
  }
  if (lane == 31) warp_tot[warp] = v;
  __syncthreads();
  uint32_t off = 0;
  for (int w = 0; w < warp; ++w) off += warp_tot[w];
  return v + off;
}

template <typename T>
__global__ void __launch_bounds__(kThreads, 4) s3ttmc_chain_kernel(const ChainParams p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem<T> &sm = *reinterpret_cast<Smem<T> *>(smem_raw);
  const int tid = threadIdx.x;
  const Chunk ch = p.chunks[blockIdx.x];
  if (!SPB_BOUND(ch.ob <= ch.oe && ch.oe <= p.nown && ch.row < p.nrows && (ch.slot == kDirect || ch.slot < p.nslots),
                 201, blockIdx.x))
    return;  // the whole CTA leaves
  const T *U = reinterpret_cast<const T *>(p.U);
  const T *cc = reinterpret_cast<const T *>(p.c);
  const uint32_t R = p.R, m2 = p.m2;
  const bool rows16 = R == (uint32_t)kRP && (reinterpret_cast<uintptr_t>(p.U) & 15u) == 0;

  for (uint32_t b = tid; b < m2; b += kThreads) {  // lexicographic pairs
    uint32_t x = 0, rem = b;
    while (rem >= R - x) {
      rem -= R - x;
      ++x;
    }
    sm.px[b] = (uint8_t)x;
    sm.py[b] = (uint8_t)(x + rem);
  }
  __syncthreads();
  // this thread's entries of G: rows a0, a0 + 1, columns b0 + 16 k
  const int a0 = 2 * (tid & 7), b0 = tid >> 3;
  double gsum[2][kBeta];
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int k = 0; k < kBeta; ++k) gsum[a][k] = 0.0;

  // owner records of the window [o, o + kB): thread t holds owners 2t, 2t+1;
  // the next window is fetched while the current batch is computed
  struct Rec {
    uint4 ids;
    T c;
    uint32_t f;
  };
  auto fetch = [&](uint64_t w0, Rec (&r)[2]) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const uint64_t o = w0 + (uint64_t)(2 * tid + h);
      if (o < ch.oe) {
        r[h].ids = *reinterpret_cast<const uint4 *>(p.S + o * p.sstride);
        r[h].c = cc[o];
        r[h].f = p.flags[o];
      }
    }
  };
  Rec rec[2];
  fetch(ch.ob, rec);
  for (uint64_t o0 = ch.ob; o0 < ch.oe;) {
    const uint64_t left = ch.oe - o0;
    // ---- batch: the window's owners, counts of group and subgroup starts
    // (packed: subgroup starts << 16 | group starts)
    uint32_t fl[2] = {0u, 0u};
    bool in[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int i = 2 * tid + h;
      in[h] = (uint64_t)i < left;
      if (in[h]) {
        uint4 ids = rec[h].ids;
        if (!SPB_BOUND(ids.x < p.nrows && ids.y < p.nrows && ids.z < p.nrows, 202, o0 + (uint64_t)i))
          ids = make_uint4(0, 0, 0, 0);
        sm.s1[i] = ids.x;
        sm.s2[i] = ids.y;
        sm.s3[i] = ids.z;
        sm.c[i] = rec[h].c;
        uint32_t f = rec[h].f;
        if (i == 0) f = 3u;  // a batch starts a group and a subgroup
        fl[h] = (f & 1u) | (((f >> 1) & 1u) << 16);
        // the W stage gathers this row after two barriers
        prefetch_l1(U + (uint64_t)ids.z * R);
      }
    }
    const uint32_t c1 = cta_scan(fl[0] + fl[1], sm.warp_tot);  // counts through owner 2t+1
    const uint32_t c0 = c1 - fl[1];                            // counts through owner 2t
    const uint32_t cnt[2] = {c0, c1};
    auto within = [](uint32_t c) { return (c & 0xffffu) <= (uint32_t)kG && (c >> 16) <= (uint32_t)kSG; };
    const bool v[2] = {in[0] && within(c0), in[1] && within(c1)};
    // The batch is the first nb owners (validity is a prefix: the counts
    // grow along the owners).  Exactly one thread sees the boundary: owner
    // 2t - 1 valid and 2t not, 2t valid and 2t + 1 not, or all 256 valid.
    const bool prev_valid = tid > 0 && (uint64_t)(2 * tid - 1) < left && within(c0 - fl[0]);
    if (!v[0] && prev_valid) sm.nb = 2 * tid;
    if (v[0] && !v[1]) sm.nb = 2 * tid + 1;
    if (v[1] && tid == kThreads - 1) sm.nb = kB;
    __syncthreads();
    const int nb = sm.nb;
    fetch(o0 + (uint64_t)nb, rec);  // in flight during this batch
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      if (!v[h]) continue;
      const int i = 2 * tid + h;
      const uint32_t g = cnt[h] & 0xffffu, sg = cnt[h] >> 16;
      sm.sg_of[i] = (uint8_t)(sg - 1);
      if (fl[h] >> 16) {
        sm.sg_start[sg - 1] = (uint16_t)i;
        sm.sg_s2[sg - 1] = sm.s2[i];
      }
      if (fl[h] & 0xffffu) {
        sm.g_sg[g - 1] = (uint16_t)(sg - 1);
        sm.g_s1[g - 1] = sm.s1[i];
      }
      if (i == nb - 1) {
        sm.nsg = (int)sg;
        sm.ng = (int)g;
        sm.sg_start[sg] = (uint16_t)nb;
        sm.g_sg[g] = (uint16_t)sg;
      }
    }
    __syncthreads();
    const int nsg = sm.nsg, ng = sm.ng;
    // ---- W of every subgroup.  Lane j (16 threads, one per column)
    // sums the owners [nb j / 8, nb (j + 1) / 8) in order, whatever the
    // subgroup sizes; the part of a subgroup begun in an earlier lane goes
    // to carry[j] and is added after the barrier, lanes in order.
    {
      // at R = 16 the s_2 row of every subgroup and the s_1 row of every
      // group are copied asynchronously while the W gathers run
      constexpr int kC = kRP * (int)sizeof(T) / 16, kE = 16 / (int)sizeof(T);
      if (rows16) {
        for (int e = tid; e < nsg * kC; e += kThreads) {
          const int sg = e / kC, k = e - sg * kC;
          cp_async16(&sm.u.b.U2[sg][k * kE], U + (uint64_t)sm.sg_s2[sg] * kRP + k * kE);
        }
        for (int e = tid; e < ng * kC; e += kThreads) {
          const int g = e / kC, k = e - g * kC;
          cp_async16(&sm.u.b.U1[g][k * kE], U + (uint64_t)sm.g_s1[g] * kRP + k * kE);
        }
      }
      constexpr int kLanes = kThreads / 16;
      const int x = tid & 15, j = tid >> 4;
      const int i0 = nb * j / kLanes, i1 = nb * (j + 1) / kLanes;
      const bool xin = (uint32_t)x < R;
      if (x == 0) sm.carry_sg[j] = -1;
      if (i0 < i1) {
        int cur = sm.sg_of[i0];
        bool own = sm.sg_start[cur] == i0;
        T w = T(0);
        auto flush = [&]() {
          if (own) {
            sm.u.b.W[cur][x] = w;
          } else {
            sm.carry[j][x] = w;
            if (x == 0) sm.carry_sg[j] = cur;
          }
        };
        for (int i = i0; i < i1; i += 8) {
          T uv[8];
#pragma unroll
          for (int k = 0; k < 8; ++k) uv[k] = (i + k < i1 && xin) ? U[(uint64_t)sm.s3[i + k] * R + x] : T(0);
#pragma unroll
          for (int k = 0; k < 8; ++k) {
            if (i + k >= i1) break;
            const int sg = sm.sg_of[i + k];
            if (sg != cur) {
              flush();
              w = T(0);
              cur = sg;
              own = true;
            }
            w = fma(sm.c[i + k], uv[k], w);
          }
        }
        flush();
      }
      if (rows16) {
        cp_async_wait_all();
      } else {  // the s_2 row of every subgroup and the s_1 row of every group
        for (int e = tid; e < nsg * kRP; e += kThreads) {
          const int sg = e >> 4, xx = e & 15;
          sm.u.b.U2[sg][xx] = (uint32_t)xx < R ? U[(uint64_t)sm.sg_s2[sg] * R + xx] : T(0);
        }
        for (int e = tid; e < ng * kRP; e += kThreads) {
          const int g = e >> 4, xx = e & 15;
          sm.u.b.U1[g][xx] = (uint32_t)xx < R ? U[(uint64_t)sm.g_s1[g] * R + xx] : T(0);
        }
      }
      __syncthreads();
      if (tid < kRP)
        for (int jj = 1; jj < kLanes; ++jj) {
          const int sg = sm.carry_sg[jj];
          if (sg >= 0) sm.u.b.W[sg][tid] += sm.carry[jj][tid];
        }
    }
    __syncthreads();
    // ---- Q of every group: sum over its subgroups of U2 (x)s W, one 4 x 4
    // tile of the upper block triangle per task (tiles in column order:
    // (0,0), (0,1), (1,1), (0,2), ...).  A batch of few groups splits each
    // group's subgroups into P parts (slots g P .. g P + P - 1 of Q), so that
    // one large group does not leave most threads idle; the parts are added
    // into slot g P before the G stage.
    const int P = max(1, min(kG / ng, nsg / (4 * ng)));
    {
      const int nbk = ((int)R + 3) >> 2, ntile = nbk * (nbk + 1) / 2;
      for (int e = tid; e < ng * P * ntile; e += kThreads) {
        const int gp = e / ntile, g = gp / P, part = gp - g * P;
        const int s0 = sm.g_sg[g], len = sm.g_sg[g + 1] - s0;
        int X = e - gp * ntile, Yb = 0;
        while (X > Yb) {
          X -= Yb + 1;
          ++Yb;
        }
        T q[4][4];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) q[i][j] = T(0);
        for (int sg = s0 + len * part / P; sg < s0 + len * (part + 1) / P; ++sg) {
          T ux[4], wx[4], uy[4], wy[4];
          load4(&sm.u.b.U2[sg][4 * X], ux);
          load4(&sm.u.b.W[sg][4 * X], wx);
          load4(&sm.u.b.U2[sg][4 * Yb], uy);
          load4(&sm.u.b.W[sg][4 * Yb], wy);
#pragma unroll
          for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              q[i][j] = fma(ux[i], wy[j], q[i][j]);
              q[i][j] = fma(wx[i], uy[j], q[i][j]);
            }
        }
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const uint32_t x = 4 * X + i, y = 4 * Yb + j;
            if (x <= y && y < R) sm.u.b.Q[gp][pair_index(x, y, R)] = q[i][j];
          }
      }
    }
    __syncthreads();
    if (P > 1) {
      for (int e = tid; e < ng * (int)m2; e += kThreads) {
        const int g = e / (int)m2, b = e - g * (int)m2;
        T q = sm.u.b.Q[g * P][b];
        for (int part = 1; part < P; ++part) q += sm.u.b.Q[g * P + part][b];
        sm.u.b.Q[g * P][b] = q;
      }
      __syncthreads();
    }
    // ---- G += U1 (x) Q over the batch's groups (FP64: straight into the
    // row totals; FP32: a batch sum in FP32, folded into the FP64 totals)
    if constexpr (sizeof(T) == 8) {
      for (int g = 0; g < ng; ++g) {
        const double2 u = *reinterpret_cast<const double2 *>(&sm.u.b.U1[g][a0]);
#pragma unroll
        for (int k = 0; k < kBeta; ++k) {
          const int b = b0 + 16 * k;
          const double q = b < (int)m2 ? (double)sm.u.b.Q[g * P][b] : 0.0;
          gsum[0][k] = fma(u.x, q, gsum[0][k]);
          gsum[1][k] = fma(u.y, q, gsum[1][k]);
        }
      }
    } else {
      T acc[2][kBeta];
#pragma unroll
      for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int k = 0; k < kBeta; ++k) acc[a][k] = T(0);
      for (int g = 0; g < ng; ++g) {
        const T u0 = sm.u.b.U1[g][a0], u1 = sm.u.b.U1[g][a0 + 1];
#pragma unroll
        for (int k = 0; k < kBeta; ++k) {
          const int b = b0 + 16 * k;
          const T q = b < (int)m2 ? sm.u.b.Q[g * P][b] : T(0);
          acc[0][k] += u0 * q;
          acc[1][k] += u1 * q;
        }
      }
#pragma unroll
      for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int k = 0; k < kBeta; ++k) gsum[a][k] += (double)acc[a][k];
    }
    o0 += (uint64_t)sm.nb;
    __syncthreads();
  }
  // ---- Y = Sym3(G) through shared memory (FP64)
  double *sG = reinterpret_cast<double *>(&sm.u.b.W[0][0]);  // kRP rows of stride kS2
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int k = 0; k < kBeta; ++k) {
      const int b = b0 + 16 * k;
      if (b < kM2) sG[(a0 + a) * kS2 + b] = gsum[a][k];
    }
  __syncthreads();
  T *Yrow = reinterpret_cast<T *>(p.Y) + (uint64_t)ch.row * p.m3;
  double *Prow = p.partials + (uint64_t)ch.slot * p.m3;
  for (uint32_t e = tid; e < p.m3; e += kThreads) {
    const uint32_t t3 = p.trip[e];
    const uint32_t q0 = t3 & 0xffu, q1 = (t3 >> 8) & 0xffu, q2 = t3 >> 16;
    const double y = sG[q0 * kS2 + pair_index(q1, q2, R)] + sG[q1 * kS2 + pair_index(q0, q2, R)] +
                     sG[q2 * kS2 + pair_index(q0, q1, R)];
    if (ch.slot == kDirect) Yrow[e] = (T)y;
    else Prow[e] = y;
  }
}

// ----------------------------------------------------- order 5 (L = 4)
//
// Leaf S = {s_1, s_2, s_3, s_4} in pivot order.  With the owners of a row
// sorted by (s_1, s_2):
//   T3_h = sum over the owners of h = (s_1, s_2) of c * K({s_3, s_4})  (order 2, m2)
//   T2_g = sum over the h of g = s_1 of Sym3(U[s_2], T3_h)             (order 3, m3)
//   G    = sum_g U[s_1] (x) T2_g                                        (16 x m3)
//   Y    = Sym4(G),  Sym4(G)[q0..q3] = sum_t G[q_t][q without q_t]
// with Sym3(u, T)[q0 q1 q2] = u[q0] T[q1 q2] + u[q1] T[q0 q2] + u[q2] T[q0 q1].
// On the order-5 power-law workload a row has 0.19 distinct s_1 and 0.63
// distinct (s_1, s_2) per owner: about 272 + 0.63 * 2448 + 0.19 * 13056
// FMAs per owner, against about 39,000 for the leaf-by-leaf team kernel.
// One CTA of 256 threads per work item; batches of up to kB5 owners, kH5
// (s_1, s_2) prefixes and kG5 s_1 groups.  T2 is formed per group as
// F = sum_h U[s_2] (x) T3_h (16 x m2, register tiles) and one Sym3 of F
// (T2[q0 q1 q2] = F[q0][q1 q2] + F[q1][q0 q2] + F[q2][q0 q1]), not one Sym3
// per prefix.  Each thread keeps 4 x 13 entries of G (rows 4a..4a+3,
// columns b + 64 k).
constexpr int kThreads5 = 256;
constexpr int kB5 = 128, kH5 = 48, kG5 = 12;
constexpr int kM3 = 816;                // packed order-3 entries at R = 16
constexpr int kS3 = kM3 + 1;            // shared row stride of G (odd: conflict-free column reads)
constexpr int kBeta5 = (kM3 + 63) / 64;  // 13

struct Chain5Params {
  const Chunk *chunks;
  uint32_t nchunks;
  const uint32_t *S;  // nown x 4 leaf ids in pivot order
  const void *c;
  const uint8_t *flags;
  const void *U;
  uint32_t R, m2, m3, m4;
  void *Y;            // packed rows, row stride m4
  double *partials;   // nslots x m4
  const uint2 *tri;   // m3: offsets in F of the three terms of Sym3 (o0 | o1 << 16 ; o2)
  const uint4 *quad;  // m4: q0 | q1 << 8 | q2 << 16 | q3 << 24 ; idx3 of q\q0, q\q1 ; q\q2, q\q3 (16 bits each)
  uint64_t nown;
  uint32_t nrows, nslots;
};

template <typename T> struct Smem5 {
  uint32_t s1[kB5], s2[kB5], s3[kB5], s4[kB5];
  T c[kB5];
  uint16_t h_start[kH5 + 1], g_h[kG5 + 1];
  uint32_t warp_tot[kThreads5 / 32];
  int nb, nh, ng;
  uint8_t px[kM2], py[kM2];
  uint2 tri[kM3];
  union __align__(16) {
    struct {
      T U3[kB5][kRP], U4[kB5][kRP];  // the owners' s_3 and s_4 rows
      T T3[kH5][kM2];
      T U2[kH5][kRP];
      T T2[kG5][kM3];
      T U1[kG5][kRP];
      T F[2][kRP * kS2];             // F of a group (two buffers, row stride kS2)
    } b;
    T G[kRP * kS3];                  // the row's G at the end (row stride kS3)
  } u;
};

template <typename T>
__global__ void __launch_bounds__(kThreads5, (sizeof(T) == 8 ? 1 : 2)) s3ttmc_chain5_kernel(const Chain5Params p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem5<T> &sm = *reinterpret_cast<Smem5<T> *>(smem_raw);
  const int tid = threadIdx.x;
  const Chunk ch = p.chunks[blockIdx.x];
  if (!SPB_BOUND(ch.ob <= ch.oe && ch.oe <= p.nown && ch.row < p.nrows && (ch.slot == kDirect || ch.slot < p.nslots),
                 211, blockIdx.x))
    return;
  const T *U = reinterpret_cast<const T *>(p.U);
  const T *cc = reinterpret_cast<const T *>(p.c);
  const uint32_t R = p.R, m2 = p.m2, m3 = p.m3;
  const bool rows16 = R == (uint32_t)kRP && (reinterpret_cast<uintptr_t>(p.U) & 15u) == 0;
  for (uint32_t b = tid; b < m2; b += kThreads5) {
    uint32_t x = 0, rem = b;
    while (rem >= R - x) {
      rem -= R - x;
      ++x;
    }
    sm.px[b] = (uint8_t)x;
    sm.py[b] = (uint8_t)(x + rem);
  }
  for (uint32_t e = tid; e < m3; e += kThreads5) sm.tri[e] = p.tri[e];

  // this thread's entries of G: rows a4 .. a4 + 3, columns bg + 64 k
  const int a4 = 4 * (tid & 3), bg = tid >> 2;
  T gsum[4][kBeta5];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int k = 0; k < kBeta5; ++k) gsum[a][k] = T(0);

  // owner record of window slot tid (tid < kB5), prefetched a batch ahead
  uint4 rid = make_uint4(0, 0, 0, 0);
  T rc = T(0);
  uint32_t rf = 0;
  auto fetch = [&](uint64_t w0) {
    const uint64_t o = w0 + (uint64_t)tid;
    if (tid < kB5 && o < ch.oe) {
      rid = *reinterpret_cast<const uint4 *>(p.S + o * 4);
      rc = cc[o];
      rf = p.flags[o];
    }
  };
  fetch(ch.ob);
  __syncthreads();
  for (uint64_t o0 = ch.ob; o0 < ch.oe;) {
    const uint64_t left = ch.oe - o0;
    const bool in = tid < kB5 && (uint64_t)tid < left;
    uint32_t fl = 0;
    if (in) {
      uint4 ids = rid;
      if (!SPB_BOUND(ids.x < p.nrows && ids.y < p.nrows && ids.z < p.nrows && ids.w < p.nrows, 212, o0 + tid))
        ids = make_uint4(0, 0, 0, 0);
      sm.s1[tid] = ids.x;
      sm.s2[tid] = ids.y;
      sm.s3[tid] = ids.z;
      sm.s4[tid] = ids.w;
      sm.c[tid] = rc;
      const uint32_t f = tid == 0 ? 3u : rf;  // a batch starts a group and a prefix
      fl = (f & 1u) | (((f >> 1) & 1u) << 16);
    }
    const uint32_t cnt = cta_scan(fl, sm.warp_tot);  // inclusive: groups | prefixes << 16
    auto within = [](uint32_t c) { return (c & 0xffffu) <= (uint32_t)kG5 && (c >> 16) <= (uint32_t)kH5; };
    const bool v = in && within(cnt);
    const bool prev_valid = tid > 0 && tid <= kB5 && (uint64_t)(tid - 1) < left && within(cnt - fl);
    if (!v && prev_valid) sm.nb = tid;
    if (v && tid == kB5 - 1) sm.nb = kB5;
    __syncthreads();
    const int nb = sm.nb;
    if (v) {
      const uint32_t g = cnt & 0xffffu, h = cnt >> 16;
      if (fl >> 16) sm.h_start[h - 1] = (uint16_t)tid;
      if (fl & 0xffffu) sm.g_h[g - 1] = (uint16_t)(h - 1);
      if (tid == nb - 1) {
        sm.nh = (int)h;
        sm.ng = (int)g;
        sm.h_start[h] = (uint16_t)nb;
        sm.g_h[g] = (uint16_t)h;
      }
    }
    __syncthreads();
    fetch(o0 + (uint64_t)nb);  // in flight during this batch
    const int nh = sm.nh, ng = sm.ng;
    // ---- stage the owners' s_3 / s_4 rows and the pivots' s_2 / s_1 rows;
    // at R = 16 (rows of whole 16-byte pieces) as asynchronous copies that
    // are all in flight at once
    if (rows16) {
      constexpr int kC = kRP * (int)sizeof(T) / 16;  // 16-byte pieces per row
      constexpr int kE = 16 / (int)sizeof(T);        // elements per piece
      for (int e = tid; e < nb * 2 * kC; e += kThreads5) {
        const int i = e / (2 * kC), r = e - i * 2 * kC, w = r / kC, k = r - w * kC;
        const uint32_t s = w ? sm.s4[i] : sm.s3[i];
        cp_async16(w ? &sm.u.b.U4[i][k * kE] : &sm.u.b.U3[i][k * kE], U + (uint64_t)s * kRP + k * kE);
      }
      for (int e = tid; e < nh * kC; e += kThreads5) {
        const int h = e / kC, k = e - h * kC;
        cp_async16(&sm.u.b.U2[h][k * kE], U + (uint64_t)sm.s2[sm.h_start[h]] * kRP + k * kE);
      }
      for (int e = tid; e < ng * kC; e += kThreads5) {
        const int g = e / kC, k = e - g * kC;
        cp_async16(&sm.u.b.U1[g][k * kE], U + (uint64_t)sm.s1[sm.h_start[sm.g_h[g]]] * kRP + k * kE);
      }
      cp_async_wait_all();
    } else {
      for (int e = tid; e < nb * kRP; e += kThreads5) {
        const int i = e / kRP, x = e - i * kRP;
        sm.u.b.U3[i][x] = (uint32_t)x < R ? U[(uint64_t)sm.s3[i] * R + x] : T(0);
        sm.u.b.U4[i][x] = (uint32_t)x < R ? U[(uint64_t)sm.s4[i] * R + x] : T(0);
      }
      for (int e = tid; e < nh * kRP; e += kThreads5) {
        const int h = e / kRP, x = e - h * kRP;
        sm.u.b.U2[h][x] = (uint32_t)x < R ? U[(uint64_t)sm.s2[sm.h_start[h]] * R + x] : T(0);
      }
      for (int e = tid; e < ng * kRP; e += kThreads5) {
        const int g = e / kRP, x = e - g * kRP;
        sm.u.b.U1[g][x] = (uint32_t)x < R ? U[(uint64_t)sm.s1[sm.h_start[sm.g_h[g]]] * R + x] : T(0);
      }
    }
    __syncthreads();
    // ---- T3 of every prefix h: one thread per (h, x), the row x of T3
    for (int e = tid; e < nh * kRP; e += kThreads5) {
      const int h = e / kRP, x = e - h * kRP;
      if ((uint32_t)x >= R) continue;
      T acc[kRP];
#pragma unroll
      for (int y = 0; y < kRP; ++y) acc[y] = T(0);
      for (int i = sm.h_start[h]; i < sm.h_start[h + 1]; ++i) {
        const T c = sm.c[i], a3 = c * sm.u.b.U3[i][x], a4 = c * sm.u.b.U4[i][x];
#pragma unroll
        for (int y = 0; y < kRP; ++y) acc[y] += a3 * sm.u.b.U4[i][y] + a4 * sm.u.b.U3[i][y];
      }
      // row x of the packed order-2 tensor: entries (x, y), y >= x
      const uint32_t base = (uint32_t)x * R - ((uint32_t)x * (uint32_t)(x - 1)) / 2;
#pragma unroll
      for (int y = 0; y < kRP; ++y)
        if (y >= x && (uint32_t)y < R) sm.u.b.T3[h][base + (uint32_t)(y - x)] = acc[y];
    }
    __syncthreads();
    // ---- T2 of every group g, one group at a time:
    //   F_g = sum over its prefixes h of U2_h (x) T3_h    (16 x m2; rows
    //         r4 .. r4 + 3 and columns c + 64 j of it per thread)
    //   T2_g[q0 q1 q2] = F_g[q0][q1 q2] + F_g[q1][q0 q2] + F_g[q2][q0 q1]
    // F alternates between two buffers, so one barrier per group suffices.
    {
      const int r4 = 4 * (tid & 3), c0 = tid >> 2;
      for (int g = 0; g < ng; ++g) {
        T f[4][3];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int j = 0; j < 3; ++j) f[a][j] = T(0);
        for (int h = sm.g_h[g]; h < sm.g_h[g + 1]; ++h) {
          T u[4], t[3];
          load4(&sm.u.b.U2[h][r4], u);
#pragma unroll
          for (int j = 0; j < 3; ++j) {
            const int col = c0 + 64 * j;
            t[j] = col < (int)m2 ? sm.u.b.T3[h][col] : T(0);
          }
#pragma unroll
          for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int j = 0; j < 3; ++j) f[a][j] = fma(u[a], t[j], f[a][j]);
        }
        T *F = sm.u.b.F[g & 1];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int j = 0; j < 3; ++j) {
            const int col = c0 + 64 * j;
            if (col < kM2) F[(r4 + a) * kS2 + col] = f[a][j];
          }
        __syncthreads();
        for (int e = tid; e < (int)m3; e += kThreads5) {
          const uint2 o = sm.tri[e];
          sm.u.b.T2[g][e] = F[o.x & 0xffffu] + F[o.x >> 16] + F[o.y];
        }
      }
    }
    __syncthreads();
    // ---- G += U1_g (x) T2_g over the batch's groups
    for (int g = 0; g < ng; ++g) {
      T u[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) u[a] = sm.u.b.U1[g][a4 + a];
#pragma unroll
      for (int k = 0; k < kBeta5; ++k) {
        const int b = bg + 64 * k;
        const T t2 = b < (int)m3 ? sm.u.b.T2[g][b] : T(0);
#pragma unroll
        for (int a = 0; a < 4; ++a) gsum[a][k] += u[a] * t2;
      }
    }
    o0 += (uint64_t)nb;
    __syncthreads();
  }
  // ---- Y = Sym4(G) through shared memory
  T *sG = sm.u.G;  // kRP rows of stride kS3
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int k = 0; k < kBeta5; ++k) {
      const int b = bg + 64 * k;
      if (b < kM3) sG[(a4 + a) * kS3 + b] = gsum[a][k];
    }
  __syncthreads();
  T *Yrow = reinterpret_cast<T *>(p.Y) + (uint64_t)ch.row * p.m4;
  double *Prow = p.partials + (uint64_t)ch.slot * p.m4;
  for (uint32_t e = tid; e < p.m4; e += kThreads5) {
    const uint4 qd = p.quad[e];
    const uint32_t q0 = qd.x & 0xffu, q1 = (qd.x >> 8) & 0xffu, q2 = (qd.x >> 16) & 0xffu, q3 = qd.x >> 24;
    const double y = (double)sG[q0 * kS3 + (qd.y & 0xffffu)] + (double)sG[q1 * kS3 + (qd.y >> 16)] +
                     (double)sG[q2 * kS3 + (qd.z & 0xffffu)] + (double)sG[q3 * kS3 + (qd.z >> 16)];
    if (ch.slot == kDirect) Yrow[e] = (T)y;
    else Prow[e] = y;
  }
}

// ---------------------------------------------------------------- build

__global__ void degree_kernel(const uint32_t *inds0, uint64_t n, uint32_t *deg) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    atomicAdd(&deg[inds0[i]], 1u);
}

__global__ void desc_key_kernel(const uint32_t *deg, uint32_t n, uint32_t *key) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) key[i] = ~deg[i];  // ascending key = descending degree
}

__global__ void rank_kernel(const uint32_t *by_degree, uint32_t n, uint32_t *rank) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) rank[by_degree[k]] = k;
}

// row of every owner: the last i with row_ptr[i] <= o
__global__ void owner_row_kernel(const uint64_t *row_ptr, uint32_t dim, uint64_t nown, uint32_t *own_row) {
  const uint64_t o = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= nown) return;
  uint32_t lo = 0, hi = dim;  // row_ptr[lo] <= o < row_ptr[hi]
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (row_ptr[mid] <= o) lo = mid; else hi = mid;
  }
  own_row[o] = lo;
}

// Leaf ids in pivot order (ascending degree rank) and the sort key of the
// first L-1 pivots (most significant first).
__global__ void pivot_order_kernel(const uint32_t *S, uint64_t nown, uint32_t sstride, uint32_t L, const uint32_t *rank,
                                   int bits, uint32_t *S_out, uint64_t *key) {
  const uint64_t o = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= nown) return;
  uint32_t id[8], rk[8];
  for (uint32_t k = 0; k < L; ++k) {
    id[k] = S[o * sstride + k];
    rk[k] = rank[id[k]];
  }
  for (uint32_t a = 1; a < L; ++a) {  // insertion sort by rank
    const uint32_t vi = id[a], vr = rk[a];
    int b = (int)a - 1;
    while (b >= 0 && rk[b] > vr) {
      id[b + 1] = id[b];
      rk[b + 1] = rk[b];
      --b;
    }
    id[b + 1] = vi;
    rk[b + 1] = vr;
  }
  uint64_t kv = 0;
  for (uint32_t k = 0; k + 1 < L; ++k) kv = (kv << bits) | rk[k];
  key[o] = kv;
  for (uint32_t k = 0; k < sstride; ++k) S_out[o * sstride + k] = k < L ? id[k] : 0u;
}

__global__ void gather_rows_kernel(const uint32_t *perm, const uint32_t *own_row, uint64_t n, uint32_t *out) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = own_row[perm[i]];
}

__global__ void chain_gather_kernel(const uint32_t *perm, uint64_t nown, uint32_t sstride, const uint32_t *S_in,
                                    const double *c_in, uint32_t *S_out, double *c64, float *c32) {
  const uint64_t o = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= nown) return;
  const uint32_t src = perm[o];
  for (uint32_t k = 0; k < sstride; ++k) S_out[o * sstride + k] = S_in[(uint64_t)src * sstride + k];
  c64[o] = c_in[src];
  c32[o] = (float)c_in[src];
}

// bit k: owner o starts a new prefix of k + 1 pivots (a new row starts all)
__global__ void chain_flags_kernel(const uint32_t *S, const uint32_t *row_sorted, uint64_t nown, uint32_t sstride,
                                   uint32_t L, uint8_t *flags) {
  const uint64_t o = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= nown) return;
  uint32_t f = 0;
  if (o == 0 || row_sorted[o] != row_sorted[o - 1]) {
    f = 0xffu;
  } else {
    bool differ = false;
    for (uint32_t k = 0; k + 1 < L; ++k) {
      differ = differ || S[o * sstride + k] != S[(o - 1) * sstride + k];
      if (differ) f |= 1u << k;
    }
  }
  flags[o] = (uint8_t)f;
}

inline unsigned blocks_for(uint64_t n, unsigned b) { return (unsigned)std::max<uint64_t>(1, (n + b - 1) / b); }

}  // namespace
uint64_t chain_light_max(const TensorState &t);
namespace {

template <class V> void upload(DBuf<V> &d, const std::vector<V> &h) {
  d.alloc(h.size());
  if (!h.empty()) SPB_CUDA(cudaMemcpy(d.p, h.data(), h.size() * sizeof(V), cudaMemcpyHostToDevice));
}

uint64_t heavy_owner_count(const TensorState &t) {
  uint64_t s = 0;
  for (uint32_t i = 0; i < t.dim; ++i) {
    const uint64_t c = t.h_row_ptr[i + 1] - t.h_row_ptr[i];
    if (c > chain_light_max(t)) s += c;
  }
  return s;
}

// Items of rows [r0, r1) in row order: rows of at most chain_light_max owners
// as one light item each, heavier rows as chain items of at most co owners
// (a row of several items gets partial-sum slots).  Returns the slot count.
uint32_t cut_chain_rows(const TensorState &t, uint64_t co, uint32_t r0, uint32_t r1, std::vector<Chunk> &ch,
                        std::vector<SplitRow> &sp, std::vector<Chunk> &lt) {
  ch.clear();
  sp.clear();
  lt.clear();
  uint32_t slot = 0;
  for (uint32_t i = r0; i < r1; ++i) {
    const uint64_t b = t.h_row_ptr[i], e = t.h_row_ptr[(size_t)i + 1];
    if (e - b <= chain_light_max(t)) {
      lt.push_back(Chunk{i, kDirect, b, e});
    } else if (e - b <= co) {
      ch.push_back(Chunk{i, kDirect, b, e});
    } else {
      const uint32_t s0 = slot;
      for (uint64_t x = b; x < e; x += co) ch.push_back(Chunk{i, slot++, x, std::min(e, x + co)});
      sp.push_back(SplitRow{i, s0, slot, 0});
    }
  }
  return slot;
}

}  // namespace

bool chain_supported(const TensorState &t, uint32_t R) {
  return (t.order == 4 || t.order == 5) && R >= 1 && R <= (uint32_t)kRP && t.dim < (1u << 21) &&
         t.nown < (1ull << 32);
}

uint64_t chain_light_max(const TensorState &t) { return t.order == 4 ? kChainLight : 0; }

ChainData &chain_data(TensorState &t) {
  if (t.chain) return *t.chain;
  NvtxRange nv("chain build");
  auto cd = std::make_shared<ChainData>();
  const uint32_t L = t.order - 1, n = t.dim;
  const uint64_t nown = t.nown;
  cd->L = L;
  cudaStream_t st = 0;
  // degree rank of every node (0 = most frequent; ties by id)
  DBuf<uint32_t> deg(n), key(n), key_sorted(n), ids(n), by_degree(n), rank(n);
  SPB_CUDA(cudaMemsetAsync(deg.p, 0, sizeof(uint32_t) * n, st));
  if (t.nnz) {
    degree_kernel<<<blocks_for(t.nnz * t.order, 256), 256, 0, st>>>(t.inds.p, t.nnz * t.order, deg.p);
    SPB_LAUNCH_CHECK();
  }
  desc_key_kernel<<<blocks_for(n, 256), 256, 0, st>>>(deg.p, n, key.p);
  SPB_LAUNCH_CHECK();
  device_iota(ids.p, n, st);
  {
    size_t tmp = 0;
    SPB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, key.p, key_sorted.p, ids.p, by_degree.p, n, 0, 32, st));
    DBuf<char> work(std::max<size_t>(tmp, 1));
    SPB_CUDA(cub::DeviceRadixSort::SortPairs(work.p, tmp, key.p, key_sorted.p, ids.p, by_degree.p, n, 0, 32, st));
  }
  rank_kernel<<<blocks_for(n, 256), 256, 0, st>>>(by_degree.p, n, rank.p);
  SPB_LAUNCH_CHECK();
  deg.release();
  key.release();
  key_sorted.release();
  ids.release();
  by_degree.release();

  // owners: leaves in pivot order; stable sort by the pivot key, then by row
  const int bits = bits_for(n ? n - 1 : 0);
  const int key_bits = bits * (int)(L - 1);
  if (key_bits > 64) fail(SYMPROP_ERR_SIZE, "chain schedule: pivot key of %d bits", key_bits);
  DBuf<uint32_t> S_piv(nown * t.sstride), own_row(nown), perm_a(nown), perm_b(nown), rows_a(nown), rows_b(nown);
  DBuf<uint64_t> pkey(nown), pkey_sorted(nown);
  if (nown) {
    pivot_order_kernel<<<blocks_for(nown, 256), 256, 0, st>>>(t.own_S.p, nown, t.sstride, L, rank.p, bits, S_piv.p,
                                                               pkey.p);
    SPB_LAUNCH_CHECK();
    owner_row_kernel<<<blocks_for(nown, 256), 256, 0, st>>>(t.row_ptr.p, n, nown, own_row.p);
    SPB_LAUNCH_CHECK();
    device_iota(perm_a.p, nown, st);
    size_t tmp1 = 0, tmp2 = 0;
    SPB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp1, pkey.p, pkey_sorted.p, perm_a.p, perm_b.p, nown, 0,
                                             std::max(key_bits, 1), st));
    SPB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp2, rows_a.p, rows_b.p, perm_b.p, perm_a.p, nown, 0,
                                             bits_for(n), st));
    DBuf<char> work(std::max<size_t>(std::max(tmp1, tmp2), 1));
    SPB_CUDA(cub::DeviceRadixSort::SortPairs(work.p, tmp1, pkey.p, pkey_sorted.p, perm_a.p, perm_b.p, nown, 0,
                                             std::max(key_bits, 1), st));
    gather_rows_kernel<<<blocks_for(nown, 256), 256, 0, st>>>(perm_b.p, own_row.p, nown, rows_a.p);
    SPB_LAUNCH_CHECK();
    SPB_CUDA(cub::DeviceRadixSort::SortPairs(work.p, tmp2, rows_a.p, rows_b.p, perm_b.p, perm_a.p, nown, 0,
                                             bits_for(n), st));
  }
  cd->S.alloc(nown * t.sstride);
  cd->c64.alloc(nown);
  cd->c32.alloc(nown);
  cd->flags.alloc(nown);
  if (nown) {
    chain_gather_kernel<<<blocks_for(nown, 256), 256, 0, st>>>(perm_a.p, nown, t.sstride, S_piv.p, t.own_c64.p, cd->S.p,
                                                               cd->c64.p, cd->c32.p);
    SPB_LAUNCH_CHECK();
    chain_flags_kernel<<<blocks_for(nown, 256), 256, 0, st>>>(cd->S.p, rows_b.p, nown, t.sstride, L, cd->flags.p);
    SPB_LAUNCH_CHECK();
  }
  // work items: the rows' owner ranges are unchanged (the sort keeps rows);
  // light rows one item each, heavy rows cut into items of at most co owners
  const uint64_t heavy_owners = heavy_owner_count(t);
  const uint64_t target_items = 148ull * 4ull * 8ull;
  uint64_t co = (heavy_owners + target_items - 1) / target_items;
  co = std::min<uint64_t>(std::max<uint64_t>(co, 256), 1024);
  cd->chunk_owners = (uint32_t)co;
  std::vector<Chunk> ch, lt;
  std::vector<SplitRow> sp;
  cd->nslots = cut_chain_rows(t, co, 0, t.dim, ch, sp, lt);
  sort_heaviest_first(ch, 0, ch.size(), co);
  sort_heaviest_first(lt, 0, lt.size(), kChainLight);
  cd->nchunks = (uint32_t)ch.size();
  cd->nsplit = (uint32_t)sp.size();
  cd->nlight = (uint32_t)lt.size();
  upload(cd->chunks, ch);
  upload(cd->split, sp);
  upload(cd->light, lt);
  SPB_CUDA(cudaDeviceSynchronize());
  t.chain = cd;
  return *cd;
}

const RowBands &chain_bands(TensorState &t, uint32_t nb) {
  ChainData &cd = chain_data(t);
  nb = std::max<uint32_t>(1, std::min<uint32_t>(nb, std::max<uint32_t>(t.dim, 1)));
  auto found = cd.bands.find(nb);
  if (found != cd.bands.end()) return *found->second;
  auto b = std::make_unique<RowBands>();
  b->nb = nb;
  std::vector<Chunk> ch, lt;
  std::vector<SplitRow> sp;
  cut_chain_rows(t, cd.chunk_owners, 0, t.dim, ch, sp, lt);
  b->row0.resize(nb + 1);
  b->chunk0.resize(nb + 1);
  b->split0.resize(nb + 1);
  b->light0.resize(nb + 1);
  for (uint32_t k = 0; k <= nb; ++k) {
    const uint32_t r = (uint32_t)((uint64_t)t.dim * k / nb);
    b->row0[k] = r;
    auto before = [r](const auto &v) {
      return (uint32_t)(std::lower_bound(v.begin(), v.end(), r, [](const auto &c, uint32_t x) { return c.row < x; }) -
                        v.begin());
    };
    b->chunk0[k] = before(ch);
    b->split0[k] = before(sp);
    b->light0[k] = before(lt);
  }
  for (uint32_t k = 0; k < nb; ++k) {
    sort_heaviest_first(ch, b->chunk0[k], b->chunk0[k + 1], cd.chunk_owners);
    sort_heaviest_first(lt, b->light0[k], b->light0[k + 1], kChainLight);
  }
  upload(b->chunks, ch);
  upload(b->split, sp);
  upload(b->light, lt);
  return *(cd.bands[nb] = std::move(b));
}

namespace {
// lexicographic sorted triples of [0, R), packed 8 bits each (per R, kept)
const uint32_t *triples(uint32_t R) {
  static std::mutex mu;
  // kept for the life of the process (a few KB per rank and device)
  static std::map<std::pair<int, uint32_t>, uint32_t *> cache;
  int dev = 0;
  SPB_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  uint32_t *&slot = cache[{dev, R}];
  if (!slot) {
    std::vector<uint32_t> h;
    for_each_sorted(R, 3, [&](const std::vector<uint32_t> &q, uint64_t) { h.push_back(q[0] | q[1] << 8 | q[2] << 16); });
    uint32_t *d = nullptr;
    SPB_CUDA(cudaMalloc(&d, h.size() * sizeof(uint32_t)));
    SPB_CUDA(cudaMemcpy(d, h.data(), h.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
    slot = d;
  }
  return slot;
}
}  // namespace

namespace {
// Order-5 index tables of rank R (kept per device and R): tri[e] for the
// packed order-3 entry e = (q0 <= q1 <= q2): the offsets in the 16 x kS2
// array F of (q0, (q1 q2)), (q1, (q0 q2)) and (q2, (q0 q1)), order-2
// entries packed; quad[e] for the packed order-4 entry
// (q0 <= .. <= q3): the q's and the packed order-3 indices of the four
// triples that leave one q out.
struct Order5Tables {
  uint2 *tri = nullptr;
  uint4 *quad = nullptr;
};

const Order5Tables &order5_tables(uint32_t R) {
  static std::mutex mu;
  static std::map<std::pair<int, uint32_t>, Order5Tables> cache;  // kept for the process
  int dev = 0;
  SPB_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  Order5Tables &tb = cache[{dev, R}];
  if (tb.tri) return tb;
  std::vector<int> pidx(R * R, -1), tidx(R * R * R, -1);
  for_each_sorted(R, 2, [&](const std::vector<uint32_t> &q, uint64_t lin) { pidx[q[0] * R + q[1]] = (int)lin; });
  for_each_sorted(R, 3, [&](const std::vector<uint32_t> &q, uint64_t lin) {
    tidx[(q[0] * R + q[1]) * R + q[2]] = (int)lin;
  });
  auto P = [&](uint32_t a, uint32_t b) { return (uint32_t)pidx[a * R + b]; };
  auto Tr = [&](uint32_t a, uint32_t b, uint32_t c) { return (uint32_t)tidx[(a * R + b) * R + c]; };
  std::vector<uint2> tri;
  for_each_sorted(R, 3, [&](const std::vector<uint32_t> &q, uint64_t) {
    const uint32_t o0 = q[0] * kS2 + P(q[1], q[2]), o1 = q[1] * kS2 + P(q[0], q[2]), o2 = q[2] * kS2 + P(q[0], q[1]);
    tri.push_back(make_uint2(o0 | o1 << 16, o2));
  });
  std::vector<uint4> quad;
  for_each_sorted(R, 4, [&](const std::vector<uint32_t> &q, uint64_t) {
    quad.push_back(make_uint4(q[0] | q[1] << 8 | q[2] << 16 | q[3] << 24,
                              Tr(q[1], q[2], q[3]) | Tr(q[0], q[2], q[3]) << 16,
                              Tr(q[0], q[1], q[3]) | Tr(q[0], q[1], q[2]) << 16, 0u));
  });
  SPB_CUDA(cudaMalloc(&tb.tri, tri.size() * sizeof(uint2)));
  SPB_CUDA(cudaMemcpy(tb.tri, tri.data(), tri.size() * sizeof(uint2), cudaMemcpyHostToDevice));
  SPB_CUDA(cudaMalloc(&tb.quad, quad.size() * sizeof(uint4)));
  SPB_CUDA(cudaMemcpy(tb.quad, quad.data(), quad.size() * sizeof(uint4), cudaMemcpyHostToDevice));
  return tb;
}

void chain5_launch(const TensorState &t, const ChainData &cd, const ItemSet &items, const void *dU, uint32_t R,
                   void *dYpacked, int precision, cudaStream_t st) {
  const Order5Tables &tb = order5_tables(R);
  Chain5Params p;
  p.chunks = items.chunks;
  p.nchunks = items.nchunks;
  p.S = cd.S.p;
  p.c = precision == SYMPROP_FP64 ? (const void *)cd.c64.p : (const void *)cd.c32.p;
  p.flags = cd.flags.p;
  p.U = dU;
  p.R = R;
  p.m2 = R * (R + 1) / 2;
  p.m3 = (uint32_t)symsize(R, 3);
  p.m4 = (uint32_t)symsize(R, 4);
  p.Y = dYpacked;
  p.partials = t.partials.p;
  p.tri = tb.tri;
  p.quad = tb.quad;
  p.nown = t.nown;
  p.nrows = t.dim;
  p.nslots = cd.nslots;
  if (precision == SYMPROP_FP64) {
    const size_t smem = sizeof(Smem5<double>);
    SPB_CUDA(cudaFuncSetAttribute(s3ttmc_chain5_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem));
    s3ttmc_chain5_kernel<double><<<items.nchunks, kThreads5, smem, st>>>(p);
  } else {
    const size_t smem = sizeof(Smem5<float>);
    SPB_CUDA(cudaFuncSetAttribute(s3ttmc_chain5_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem));
    s3ttmc_chain5_kernel<float><<<items.nchunks, kThreads5, smem, st>>>(p);
  }
  SPB_LAUNCH_CHECK();
  spb_check_host(st, "S3TTMc chain kernel (order 5)");
}
}  // namespace

void chain_launch(const TensorState &t, const ChainData &cd, const ItemSet &items, const void *dU, uint32_t R,
                  void *dYpacked, int precision, cudaStream_t st) {
  if (!chain_supported(t, R)) fail(SYMPROP_ERR_SIZE, "chain S3TTMc does not support order %u rank %u", t.order, R);
  if (!items.nchunks) return;
  if (t.order == 5) {
    chain5_launch(t, cd, items, dU, R, dYpacked, precision, st);
    return;
  }
  ChainParams p;
  p.chunks = items.chunks;
  p.nchunks = items.nchunks;
  p.S = cd.S.p;
  p.sstride = t.sstride;
  p.c = precision == SYMPROP_FP64 ? (const void *)cd.c64.p : (const void *)cd.c32.p;
  p.flags = cd.flags.p;
  p.U = dU;
  p.R = R;
  p.m2 = R * (R + 1) / 2;
  p.m3 = (uint32_t)symsize(R, 3);
  p.Y = dYpacked;
  p.partials = t.partials.p;
  p.trip = triples(R);
  p.nown = t.nown;
  p.nrows = t.dim;
  p.nslots = cd.nslots;
  if (precision == SYMPROP_FP64) {
    const size_t smem = sizeof(Smem<double>);
    SPB_CUDA(cudaFuncSetAttribute(s3ttmc_chain_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    s3ttmc_chain_kernel<double><<<items.nchunks, kThreads, smem, st>>>(p);
  } else {
    const size_t smem = sizeof(Smem<float>);
    SPB_CUDA(cudaFuncSetAttribute(s3ttmc_chain_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    s3ttmc_chain_kernel<float><<<items.nchunks, kThreads, smem, st>>>(p);
  }
  SPB_LAUNCH_CHECK();
  spb_check_host(st, "S3TTMc chain kernel");
}

}  // namespace spb
