// S3TTMc, warp-per-owner schedule (default when the packed output fits in
// the registers of one warp: up to 4 output tiles of 4 x 4 per lane, e.g.
// order 4 / R <= 16, order 5 / R <= 10, order 6 / R <= 8).
//
// Same mathematics as the reference's level sweep
// (CompressedDTree::kronecker_product_opt5, src/compressed_dtree.cpp:421-518;
// SymOuterProd, include/detail/dense/symtensor.hpp:24-39):
//     Y[i] += c * K(S),  K(S) = sum_k K(S \ s_k) (x) U[s_k].
// A warp streams owners (tree leaves) of one row, one leaf per step, with no
// CTA barrier inside the loop:
//   * lanes stage the leaf's N-1 U rows (and c * U rows) in warp-private
//     shared memory;
//   * levels 2..N-3 of the recursion are built in warp-private shared memory
//     (colexicographic order, see s3ttmc_tiled.cu);
//   * the last level is never stored: for each of its 4 x 4 output tiles a
//     lane evaluates the N-1 parent tensors K(S \ s_k) at the tile's 4 rows
//     from level N-3 and U in registers, then adds the rank-(N-1) product
//     with the c * U rows.
// Work items (a row, or a slice of a long row) with at most kLightOwners
// owners take one warp each and are written straight from registers; larger
// ones take the 4 warps of a CTA, whose tiles are added in warp order
// (deterministic).  For a fixed prefix p the outputs (p, x), x >= last(p),
// are consecutive in the reference's lexicographic packed order, so a tile
// row is written at a precomputed row offset + x (no permutation table).
// FP32 mode folds the lane's plain FP32 sums into a Kahan-compensated
// accumulator every 4 owners.
#include <algorithm>

#include "s3ttmc_warp.cuh"

namespace spb {
namespace {

constexpr int kWarps = 4, kThreads = kWarps * 32, kMaxL = 7, kMaxNTL = 4;
constexpr uint32_t kURow = 0x80000000u;
constexpr uint32_t kPadRow = 0xffffffffu;

struct WDesc {
  uint32_t dst, nterm;
  uint32_t src[kMaxL], k[kMaxL];
};

struct WarpParams {
  const Chunk *chunks;
  uint32_t nchunks, nheavy;
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
  uint32_t m[kMaxL + 1], m4[kMaxL + 1];
  uint32_t pair_src[kMaxL * kMaxL];  // level N-3 tensor of the positions other than {k,t}
  const int4 *tiles;                 // per tile: (first row r0 inside block j, j, first column x0, 0)
  const uint4 *rowoff;               // per tile: lex offset - j of its 4 rows, or kPadRow
  uint32_t ntiles;
  uint32_t wsz;                      // per-warp staging elements: 2*L*R4 + ksz4
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

template <typename T> constexpr int min_blocks() { return sizeof(T) == 8 ? 3 : 2; }

template <int L, int NTL, typename T>
__global__ void __launch_bounds__(kThreads, min_blocks<T>()) s3ttmc_warp_kernel(const WarpParams p) {
  constexpr bool kExact = sizeof(T) == 8;
  extern __shared__ __align__(16) unsigned char smem[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t R = p.R, R4 = p.R4;

  size_t off = 0;
  uint32_t *sStart = reinterpret_cast<uint32_t *>(smem + off);
  off += (((size_t)(L + 1) * (R + 1) * 4) + 15) / 16 * 16;
  uint8_t *sJ = smem + off;
  off += ((size_t)p.jtab_len + 15) / 16 * 16;
  WDesc *sDesc = reinterpret_cast<WDesc *>(smem + off);
  off += ((size_t)p.ndesc * sizeof(WDesc) + 15) / 16 * 16;
  T *sWarp = reinterpret_cast<T *>(smem + off);  // kWarps x wsz, later the reduction area

  if constexpr (L >= 4) {
    for (uint32_t i = tid; i < (uint32_t)(L + 1) * (R + 1); i += kThreads) sStart[i] = p.starts[i];
    for (uint32_t i = tid; i < p.jtab_len; i += kThreads) sJ[i] = p.jtab[i];
    const uint32_t *src = reinterpret_cast<const uint32_t *>(p.desc);
    uint32_t *dst = reinterpret_cast<uint32_t *>(sDesc);
    const uint32_t words = p.ndesc * (uint32_t)(sizeof(WDesc) / 4);
    for (uint32_t i = tid; i < words; i += kThreads) dst[i] = src[i];
    __syncthreads();
  }

  // work item: heavy items take the whole CTA, light ones one warp each
  const bool heavy = blockIdx.x < p.nheavy;
  const uint32_t item = heavy ? blockIdx.x : p.nheavy + (blockIdx.x - p.nheavy) * kWarps + warp;
  if (!heavy && item >= p.nchunks) return;  // light CTAs have no barrier below
  const Chunk ch = p.chunks[item];

  // this lane's tiles: 4 consecutive rows r0..r0+3 of block j (all with last
  // index j) times columns x0..x0+3
  int4 tl[NTL];
  bool live[NTL];
#pragma unroll
  for (int i = 0; i < NTL; ++i) {
    const uint32_t id = (uint32_t)lane + 32u * i;
    live[i] = id < p.ntiles;
    tl[i] = live[i] ? p.tiles[id] : make_int4(0, 0, 0, 0);
  }

  T acc[NTL][4][4], cmp[NTL][4][4], tmp[NTL][4][4];
#pragma unroll
  for (int i = 0; i < NTL; ++i)
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int c = 0; c < 4; ++c) { acc[i][a][c] = T(0); cmp[i][a][c] = T(0); tmp[i][a][c] = T(0); }

  const T *U = reinterpret_cast<const T *>(p.U);
  const T *own_c = reinterpret_cast<const T *>(p.own_c);
  T *sU = sWarp + (size_t)warp * p.wsz;
  T *sW = sU + L * R4;
  T *sK = sW + L * R4;
  int pending = 0;
  const uint32_t ostep = heavy ? kWarps : 1;

  for (uint64_t o = ch.ob + (heavy ? warp : 0); o < ch.oe; o += ostep) {
    // stage the leaf's U rows
    const uint32_t *S = p.own_S + o * p.sstride;
    const T c = own_c[o];
    for (uint32_t i = lane; i < (uint32_t)L * R4; i += 32) {
      const uint32_t k = i / R4, x = i - k * R4;
      T u = T(0);
      if (x < R) u = U[(uint64_t)S[k] * R + x];
      sU[i] = u;
      sW[i] = c * u;
    }
    __syncwarp();
    // levels 2 .. L-2 in warp shared memory
    if constexpr (L >= 4) {
#pragma unroll 1
      for (int d = 2; d <= L - 2; ++d) {
        const uint32_t md = p.m[d], md4 = p.m4[d], nd = p.desc_count[d];
        const uint8_t *jt = sJ + p.jtab_off[d];
        const uint32_t *stt = sStart + d * (R + 1);
        const WDesc *dd = sDesc + p.desc_begin[d];
        for (uint32_t it = lane; it < nd * md4; it += 32) {
          const uint32_t mi = it / md4, e = it - mi * md4;
          T v = T(0);
          if (e < md) {
            const uint32_t j = jt[e], r = e - stt[j];
            const WDesc &ds = dd[mi];
#pragma unroll
            for (int t = 0; t < kMaxL; ++t) {
              if (t >= d) break;
              const uint32_t s = ds.src[t];
              const T a = (s & kURow) ? sU[(s & 0xffu) * R4 + r] : sK[s + r];
              v += a * sU[ds.k[t] * R4 + j];
            }
          }
          sK[dd[mi].dst + e] = v;
        }
        __syncwarp();
      }
    }
    // last level: the parents K(S \ s_k) at rows (r0+q, j) are
    //   sum_{t != k} K(S \ {s_k, s_t})[r0+q] * U[s_t][j]
    // (level N-3 tensors, or U rows for order 4), then the tile gets
    // sum_k A_k[q] * (c U[s_k])[x0 + cc]
#pragma unroll
    for (int i = 0; i < NTL; ++i) {
      if (!live[i]) continue;
      const uint32_t r0 = (uint32_t)tl[i].x, jt = (uint32_t)tl[i].y, x0 = (uint32_t)tl[i].z;
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
            T kv[4];
            if constexpr (L == 3) ld4(sU + (s & 0xffu) * R4 + r0, kv);
            else ld4(sK + s + r0, kv);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              A[k][q] += kv[q] * uj[t];
              A[t][q] += kv[q] * uj[k];
            }
          }
      }
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) {
          T s = T(0);
#pragma unroll
          for (int k = 0; k < L; ++k) s += A[k][q] * w[k][cc];
          if constexpr (kExact) acc[i][q][cc] += s;
          else tmp[i][q][cc] += s;
        }
    }
    if constexpr (!kExact) {
      if (++pending == 4) {
        pending = 0;
#pragma unroll
        for (int i = 0; i < NTL; ++i)
#pragma unroll
          for (int q = 0; q < 4; ++q)
#pragma unroll
            for (int cc = 0; cc < 4; ++cc) {
              T y = tmp[i][q][cc] - cmp[i][q][cc];
              T s2 = acc[i][q][cc] + y;
              cmp[i][q][cc] = (s2 - acc[i][q][cc]) - y;
              acc[i][q][cc] = s2;
              tmp[i][q][cc] = T(0);
            }
      }
    }
    __syncwarp();
  }
  if constexpr (!kExact) {
#pragma unroll
    for (int i = 0; i < NTL; ++i)
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) {
          T y = tmp[i][q][cc] - cmp[i][q][cc];
          T s2 = acc[i][q][cc] + y;
          cmp[i][q][cc] = (s2 - acc[i][q][cc]) - y;
          acc[i][q][cc] = s2 - cmp[i][q][cc];
        }
  }

  T *Yrow = reinterpret_cast<T *>(p.Y) + (uint64_t)ch.row * p.ldy;
  double *Prow = p.partials + (uint64_t)ch.slot * p.mL;
  if (!heavy) {  // one warp owns the whole work item: write from registers
#pragma unroll
    for (int i = 0; i < NTL; ++i) {
      if (!live[i]) continue;
      const uint4 ro = p.rowoff[(uint32_t)lane + 32u * i];
      const uint32_t rof[4] = {ro.x, ro.y, ro.z, ro.w};
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        if (rof[q] == kPadRow) continue;
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) {
          const uint32_t x = (uint32_t)tl[i].z + cc;
          if (x >= R || x < (uint32_t)tl[i].y) continue;
          const uint32_t qo = rof[q] + x;
          if (ch.slot == kDirect) Yrow[qo] = acc[i][q][cc];
          else Prow[qo] = (double)acc[i][q][cc];
        }
      }
    }
    return;
  }
  // heavy: add the warps' tiles in warp order
  __syncthreads();
  T *red = sWarp;  // kWarps x ntiles x 16
#pragma unroll
  for (int i = 0; i < NTL; ++i) {
    if (!live[i]) continue;
    T *dst = red + ((size_t)warp * p.ntiles + (uint32_t)lane + 32u * i) * 16;
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int cc = 0; cc < 4; ++cc) dst[q * 4 + cc] = acc[i][q][cc];
  }
  __syncthreads();
  for (uint32_t e = tid; e < p.ntiles * 16; e += kThreads) {
    const uint32_t tile = e >> 4, q = (e >> 2) & 3, cc = e & 3;
    const int4 tt = p.tiles[tile];
    const uint32_t x = (uint32_t)tt.z + cc;
    const uint4 ro = p.rowoff[tile];
    const uint32_t rof = q == 0 ? ro.x : q == 1 ? ro.y : q == 2 ? ro.z : ro.w;
    if (rof == kPadRow || x >= R || x < (uint32_t)tt.y) continue;
    T s = T(0);
#pragma unroll
    for (int w2 = 0; w2 < kWarps; ++w2) s += red[((size_t)w2 * p.ntiles + tile) * 16 + (e & 15)];
    if (ch.slot == kDirect) Yrow[rof + x] = s;
    else Prow[rof + x] = (double)s;
  }
}

}  // namespace

struct WarpPlan {
  bool ok = false;
  uint32_t L = 0, R = 0, R4 = 0, NTL = 0;
  uint32_t m[kMaxL + 1] = {}, m4[kMaxL + 1] = {};
  DBuf<uint32_t> starts;
  DBuf<uint8_t> jtab;
  uint32_t jtab_len = 0, jtab_off[kMaxL + 1] = {};
  DBuf<WDesc> desc;
  uint32_t ndesc = 0, desc_begin[kMaxL + 1] = {}, desc_count[kMaxL + 1] = {};
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
  pl->NTL = (pl->ntiles + 31) / 32;
  if (pl->NTL > (uint32_t)kMaxNTL) return pl;
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
    for (uint32_t mask = 0; mask < (1u << L); ++mask) {
      if ((uint32_t)__builtin_popcount(mask) != d) continue;
      WDesc ds{};
      ds.dst = ksz;
      offm[mask] = ksz;
      ksz += pl->m4[d];
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
  pl->ndesc = (uint32_t)desc.size();
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
    size_t work = std::max((size_t)kWarps * pl->wsz * es, (size_t)kWarps * pl->ntiles * 16 * es);
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
static void launch_w(const WarpParams &wp, uint32_t grid, size_t smem, cudaStream_t st) {
  auto kern = s3ttmc_warp_kernel<L, NTL, T>;
  SPB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kern<<<grid, kThreads, smem, st>>>(wp);
  SPB_LAUNCH_CHECK();
}

template <int L, typename T>
static void launch_w_ntl(uint32_t NTL, const WarpParams &wp, uint32_t grid, size_t smem, cudaStream_t st) {
  switch (NTL) {
    case 1: launch_w<L, 1, T>(wp, grid, smem, st); break;
    case 2: launch_w<L, 2, T>(wp, grid, smem, st); break;
    case 3: launch_w<L, 3, T>(wp, grid, smem, st); break;
    default: launch_w<L, 4, T>(wp, grid, smem, st); break;
  }
}

template <typename T>
static void launch_w_l(uint32_t L, uint32_t NTL, const WarpParams &wp, uint32_t grid, size_t smem,
                       cudaStream_t st) {
  switch (L) {
    case 2: launch_w_ntl<2, T>(NTL, wp, grid, smem, st); break;
    case 3: launch_w_ntl<3, T>(NTL, wp, grid, smem, st); break;
    case 4: launch_w_ntl<4, T>(NTL, wp, grid, smem, st); break;
    case 5: launch_w_ntl<5, T>(NTL, wp, grid, smem, st); break;
    case 6: launch_w_ntl<6, T>(NTL, wp, grid, smem, st); break;
    default: launch_w_ntl<7, T>(NTL, wp, grid, smem, st); break;
  }
}

void warp_launch(const WarpPlan &pl, const TensorState &t, const void *dU, void *dYpacked, int precision,
                 cudaStream_t st) {
  if (!t.nchunks) return;
  const int pi = precision == SYMPROP_FP64 ? 0 : 1;
  WarpParams wp{};
  wp.chunks = t.chunks.p;
  wp.nchunks = t.nchunks;
  wp.nheavy = t.nheavy;
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
    wp.m[d] = pl.m[d];
    wp.m4[d] = pl.m4[d];
  }
  for (int i = 0; i < kMaxL * kMaxL; ++i) wp.pair_src[i] = pl.pair_src[i];
  wp.tiles = pl.tiles.p;
  wp.rowoff = pl.rowoff.p;
  wp.ntiles = pl.ntiles;
  wp.wsz = pl.wsz;
  const uint32_t nlight = t.nchunks - t.nheavy;
  const uint32_t grid = t.nheavy + (nlight + kWarps - 1) / kWarps;
  if (pi == 0) launch_w_l<double>(pl.L, pl.NTL, wp, grid, pl.smem[0], st);
  else launch_w_l<float>(pl.L, pl.NTL, wp, grid, pl.smem[1], st);
}

}  // namespace spb
