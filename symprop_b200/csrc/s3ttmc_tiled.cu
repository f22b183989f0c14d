// S3TTMc, register-tiled schedule (the default for orders 3..7, R <= 64).
//
// Same mathematics as the reference's level sweep
// (CompressedDTree::kronecker_product_opt5, src/compressed_dtree.cpp:421-518;
// SymOuterProd, include/detail/dense/symtensor.hpp:24-39): for each owner
// (row i, leaf S, coefficient c) of the row-segmented owner list,
//     Y[i] += c * K(S),   K(S) = sum_k K(S \ s_k) (x) U[s_k],
// with K of every sub-multiset of S recomputed from U rows in shared memory.
//
// Layout trick: inside the kernel every packed symmetric tensor of order d is
// stored in colexicographic order (sorted by the largest index first).  The
// entries whose largest index is j then form one contiguous block
//     [C(j+d-1, d), C(j+d, d))   of length  C(j+d-1, d-1),
// and the entry (prefix p, last j) sits at C(j+d-1, d) + colex(p).  The
// symmetric outer product  out[(p, j)] = sum_k A_k[p] * B_k[j],  j >= last(p),
// is therefore a rank-L product A B^T restricted to a staircase whose column
// j is the row prefix [0, C(j+d-1, d-1)): it is computed in 4 x 4 register
// tiles with 128-bit shared loads, with no per-element index arithmetic.
// The lexicographic packed order of the reference is restored only when Y
// is written.
//
// One CTA (256 threads) per work item (a row of Y or a slice of a long row);
// owners are processed in batches of BO with L barriers per batch; when the
// output has fewer tiles than threads, G thread groups split the owners of
// each batch and are reduced once per work item.  FP32 mode folds each
// batch into a Kahan-compensated accumulator.
#include <algorithm>
#include <cstdlib>

#include "check.cuh"
#include "s3ttmc_tiled.cuh"

namespace spb {

namespace {

constexpr int kMaxLt = 7;
constexpr uint32_t kURow = 0x80000000u;
constexpr int kThreads = 256;

struct DpDesc {
  uint32_t dst;           // offset of this sub-multiset's tensor inside one owner's sK
  uint32_t nterm;
  uint32_t src[kMaxLt];   // sK offset, or kURow | position for a single id
  uint32_t k[kMaxLt];     // position whose U row multiplies the term
};

struct TiledParams {
  const Chunk *chunks;
  const uint32_t *own_S;
  const void *own_c;
  uint32_t sstride;
  const void *U;
  uint32_t R, R4;
  void *Y;
  uint64_t ldy;
  double *partials;
  uint32_t mL;
  // tables (global): starts for levels 2..L, jtab bytes, desc, tiles, lexidx
  const uint32_t *starts;   // (L+1) x (R+1): starts[d*(R+1) + j] = C(j+d-1, d)
  const uint8_t *jtab;      // concatenated jtab of levels 2..L-1
  uint32_t jtab_len;
  uint32_t jtab_off[kMaxLt + 1];
  const DpDesc *desc;
  uint32_t ndesc;
  uint32_t desc_begin[kMaxLt + 1], desc_count[kMaxLt + 1];
  uint32_t m4[kMaxLt + 1], m[kMaxLt + 1];
  uint32_t final_src[kMaxLt];
  const int2 *tiles;
  uint32_t ntiles;
  const uint32_t *lexidx;   // colex index at level L -> lexicographic packed index
  uint32_t ksz4;            // padded per-owner DP storage
  uint32_t BO, G;
  uint64_t nown;            // bounds the checked build tests
  uint32_t nrows, nslots;
};

template <typename T> struct Vec4;
template <> struct Vec4<float> {
  __device__ static void load(const float *p, float (&v)[4]) {
    float4 x = *reinterpret_cast<const float4 *>(p);
    v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
  }
};
template <> struct Vec4<double> {
  __device__ static void load(const double *p, double (&v)[4]) {
    double2 x = *reinterpret_cast<const double2 *>(p);
    double2 y = *reinterpret_cast<const double2 *>(p + 2);
    v[0] = x.x; v[1] = x.y; v[2] = y.x; v[3] = y.y;
  }
};

// number of terms of the deepest DP level (levels 2..L-1 have d terms)
__host__ __device__ constexpr int d_max(int L) { return L > 2 ? L - 1 : 1; }

template <int L, int NT, typename T>
__global__ void __launch_bounds__(kThreads, 2) s3ttmc_tiled_kernel(const TiledParams p) {
  constexpr bool kExact = sizeof(T) == 8;
  extern __shared__ __align__(16) unsigned char smem[];
  const int tid = threadIdx.x;
  const Chunk ch = p.chunks[blockIdx.x];
  if (!SPB_BOUND(ch.ob <= ch.oe && ch.oe <= p.nown && ch.row < p.nrows && (ch.slot == kDirect || ch.slot < p.nslots),
                 201, blockIdx.x))
    return;  // the whole CTA leaves (the chunk is the CTA's)
  const uint32_t R = p.R, R4 = p.R4, BO = p.BO, G = p.G;

  // ---- shared memory carve
  size_t off = 0;
  uint32_t *sStart = reinterpret_cast<uint32_t *>(smem + off);
  off += (((size_t)(L + 1) * (R + 1) * 4) + 15) / 16 * 16;
  uint8_t *sJ = smem + off;
  off += ((size_t)p.jtab_len + 15) / 16 * 16;
  DpDesc *sDesc = reinterpret_cast<DpDesc *>(smem + off);
  off += ((size_t)p.ndesc * sizeof(DpDesc) + 15) / 16 * 16;
  T *sU = reinterpret_cast<T *>(smem + off);
  T *sW = sU + (size_t)BO * L * R4;
  T *sK = sW + (size_t)BO * L * R4;

  for (uint32_t i = tid; i < (uint32_t)(L + 1) * (R + 1); i += kThreads) sStart[i] = p.starts[i];
  for (uint32_t i = tid; i < p.jtab_len; i += kThreads) sJ[i] = p.jtab[i];
  {
    const uint32_t *src = reinterpret_cast<const uint32_t *>(p.desc);
    uint32_t *dst = reinterpret_cast<uint32_t *>(sDesc);
    const uint32_t words = p.ndesc * (uint32_t)(sizeof(DpDesc) / 4);
    for (uint32_t i = tid; i < words; i += kThreads) dst[i] = src[i];
  }

  // ---- this thread's tiles and owner group
  const uint32_t ntiles = p.ntiles;
  int my_tile[NT];
  uint32_t group = 0;
  if (NT == 1) {
    group = (uint32_t)tid / max(ntiles, 1u);
    my_tile[0] = (group < G && (uint32_t)tid % max(ntiles, 1u) < ntiles) ? (int)((uint32_t)tid % ntiles) : -1;
  } else {
#pragma unroll
    for (int t = 0; t < NT; ++t) {
      uint32_t id = (uint32_t)tid + (uint32_t)t * kThreads;
      my_tile[t] = id < ntiles ? (int)id : -1;
    }
  }
  int2 tl[NT];
#pragma unroll
  for (int t = 0; t < NT; ++t) tl[t] = my_tile[t] >= 0 ? p.tiles[my_tile[t]] : make_int2(0, 0);

  T acc[NT][4][4], cmp[NT][4][4], tmp[NT][4][4];
#pragma unroll
  for (int t = 0; t < NT; ++t)
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int c = 0; c < 4; ++c) { acc[t][i][c] = T(0); cmp[t][i][c] = T(0); tmp[t][i][c] = T(0); }

  const T *U = reinterpret_cast<const T *>(p.U);
  const T *own_c = reinterpret_cast<const T *>(p.own_c);
  __syncthreads();

  for (uint64_t ob = ch.ob; ob < ch.oe; ob += BO) {
    const uint32_t nb = (uint32_t)min((uint64_t)BO, ch.oe - ob);
    // stage U rows and coefficient-scaled rows of the batch; the flat index
    // i = (o*L + k)*R4 + x advances by kThreads with carries (no division
    // inside the loop)
    const uint32_t per = L * R4;
    {
      uint32_t o = (uint32_t)tid / per, rem = (uint32_t)tid - o * per, k = rem / R4, x = rem - k * R4;
      const uint32_t dO = kThreads / per, dr = kThreads - dO * per, dK = dr / R4, dX = dr - dK * R4;
      while (o < nb) {
        const uint32_t i = o * per + k * R4 + x;
        T u = T(0);
        if (x < R) {
          const uint32_t id = p.own_S[(ob + o) * p.sstride + k];
          if (SPB_BOUND(id < p.nrows, 202, id)) u = U[(uint64_t)id * R + x];
        }
        sU[i] = u;
        sW[i] = own_c[ob + o] * u;
        x += dX;
        if (x >= R4) { x -= R4; ++k; }
        k += dK;
        if (k >= (uint32_t)L) { k -= L; ++o; }
        o += dO;
      }
    }
    __syncthreads();
    // intermediate sub-multiset tensors (colex), levels 2 .. L-1; item
    // (o, mask, e) advances by kThreads with carries
#pragma unroll 1
    for (int d = 2; d < L; ++d) {
      const uint32_t md = p.m[d], md4 = p.m4[d], nd = p.desc_count[d];
      const uint8_t *jt = sJ + p.jtab_off[d];
      const uint32_t *stt = sStart + d * (R + 1);
      const DpDesc *dd = sDesc + p.desc_begin[d];
      const uint32_t perd = nd * md4;
      uint32_t o = (uint32_t)tid / perd, rem = (uint32_t)tid - o * perd, mi = rem / md4, e = rem - mi * md4;
      const uint32_t dO = kThreads / perd, dr = kThreads - dO * perd, dM = dr / md4, dE = dr - dM * md4;
      while (o < nb) {
        const DpDesc &ds = dd[mi];
        T v = T(0);
        if (e < md) {
          const uint32_t j = jt[e];
          const uint32_t r = e - stt[j];
          const T *uo = sU + (size_t)o * per;
          const T *ko = sK + (size_t)o * p.ksz4;
#pragma unroll
          for (int t = 0; t < d_max(L); ++t) {
            if (t >= d) break;
            const uint32_t s = ds.src[t];
            const T a = (s & kURow) ? uo[(s & 0xffu) * R4 + r] : ko[s + r];
            v += a * uo[ds.k[t] * R4 + j];
          }
        }
        sK[(size_t)o * p.ksz4 + ds.dst + e] = v;
        e += dE;
        if (e >= md4) { e -= md4; ++mi; }
        mi += dM;
        if (mi >= nd) { mi -= nd; ++o; }
        o += dO;
      }
      __syncthreads();
    }
    // last level: register-tiled staircase products
    for (uint32_t o = group; o < nb; o += G) {
      const T *uo = sU + (size_t)o * per;
      const T *wo = sW + (size_t)o * per;
      const T *ko = sK + (size_t)o * p.ksz4;
#pragma unroll
      for (int k = 0; k < L; ++k) {
        const uint32_t s = p.final_src[k];
        const T *arow = (s & kURow) ? (uo + (s & 0xffu) * R4) : (ko + s);
#pragma unroll
        for (int t = 0; t < NT; ++t) {
          if (my_tile[t] < 0) continue;
          T a[4], v[4];
          Vec4<T>::load(arow + tl[t].x, a);
          Vec4<T>::load(wo + k * R4 + tl[t].y, v);
#pragma unroll
          for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int c = 0; c < 4; ++c) {
              if constexpr (kExact) acc[t][i][c] += a[i] * v[c];
              else tmp[t][i][c] += a[i] * v[c];
            }
        }
      }
    }
    if constexpr (!kExact) {
#pragma unroll
      for (int t = 0; t < NT; ++t)
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int c = 0; c < 4; ++c) {  // Kahan fold of the batch
            T y = tmp[t][i][c] - cmp[t][i][c];
            T s2 = acc[t][i][c] + y;
            cmp[t][i][c] = (s2 - acc[t][i][c]) - y;
            acc[t][i][c] = s2;
            tmp[t][i][c] = T(0);
          }
    }
    __syncthreads();
  }

  // ---- reduce owner groups (NT == 1 only), then write
  if (NT == 1 && G > 1) {
    T *red = sU;  // reuse the staging area: (G-1) x ntiles x 16
    if (group >= 1 && group < G && my_tile[0] >= 0) {
      T *dst = red + ((size_t)(group - 1) * ntiles + my_tile[0]) * 16;
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int c = 0; c < 4; ++c) dst[i * 4 + c] = acc[0][i][c] - cmp[0][i][c];
    }
    __syncthreads();
    if (group == 0 && my_tile[0] >= 0) {
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[0][i][c] -= cmp[0][i][c], cmp[0][i][c] = T(0);
      for (uint32_t g = 1; g < G; ++g) {
        const T *src = red + ((size_t)(g - 1) * ntiles + my_tile[0]) * 16;
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int c = 0; c < 4; ++c) acc[0][i][c] += src[i * 4 + c];
      }
    }
  }
  if (group != 0) return;
  const uint32_t *stL = p.starts + L * (R + 1);
#pragma unroll
  for (int t = 0; t < NT; ++t) {
    if (my_tile[t] < 0) continue;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const uint32_t j = (uint32_t)tl[t].y + c;
      if (j >= R) continue;
      const uint32_t base = stL[j], cnt = stL[j + 1] - stL[j];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const uint32_t r = (uint32_t)tl[t].x + i;
        if (r >= cnt) continue;
        const uint32_t q = p.lexidx[base + r];
        if (!SPB_BOUND(q < p.mL, 203, q)) continue;
        const T val = acc[t][i][c] - cmp[t][i][c];
        if (ch.slot == kDirect)
          reinterpret_cast<T *>(p.Y)[(uint64_t)ch.row * p.ldy + q] = val;
        else
          p.partials[(uint64_t)ch.slot * p.mL + q] = (double)val;
      }
    }
  }
}

uint64_t colex_start(uint32_t j, uint32_t d) { return symsize(j, d); }  // C(j+d-1, d)

}  // namespace

struct TiledPlan {
  uint32_t L = 0, R = 0, R4 = 0;
  uint32_t m[kMaxLt + 1] = {}, m4[kMaxLt + 1] = {};
  DBuf<uint32_t> starts, lexidx;
  DBuf<uint8_t> jtab;
  uint32_t jtab_len = 0, jtab_off[kMaxLt + 1] = {};
  DBuf<DpDesc> desc;
  uint32_t ndesc = 0, desc_begin[kMaxLt + 1] = {}, desc_count[kMaxLt + 1] = {};
  uint32_t final_src[kMaxLt] = {};
  DBuf<int2> tiles;
  uint32_t ntiles = 0;
  uint32_t ksz4 = 0;
  uint32_t BO[2] = {0, 0}, G = 1;
  int NT = 1;
  size_t smem[2] = {0, 0};
  bool ok = false;
};

std::shared_ptr<TiledPlan> tiled_plan(uint32_t N, uint32_t R) {
  auto pl = std::make_shared<TiledPlan>();
  const uint32_t L = N - 1;
  if (L < 2 || L > (uint32_t)kMaxLt || R > 64) return pl;  // not supported -> other schedule
  pl->L = L;
  pl->R = R;
  pl->R4 = (R + 3) / 4 * 4;
  for (uint32_t d = 0; d <= L; ++d) {
    pl->m[d] = (uint32_t)symsize(R, d);
    pl->m4[d] = (pl->m[d] + 3) / 4 * 4;
  }
  if (symsize(R, L) > (1u << 26)) return pl;
  // colex block starts per level
  std::vector<uint32_t> starts((size_t)(L + 1) * (R + 1), 0);
  for (uint32_t d = 1; d <= L; ++d)
    for (uint32_t j = 0; j <= R; ++j) starts[(size_t)d * (R + 1) + j] = (uint32_t)colex_start(j, d);
  // jtab for DP levels 2..L-1
  std::vector<uint8_t> jt;
  for (uint32_t d = 2; d < L; ++d) {
    pl->jtab_off[d] = (uint32_t)jt.size();
    for (uint32_t j = 0; j < R; ++j)
      for (uint32_t e = starts[(size_t)d * (R + 1) + j]; e < starts[(size_t)d * (R + 1) + j + 1]; ++e)
        jt.push_back((uint8_t)j);
  }
  pl->jtab_len = (uint32_t)jt.size();
  // DP descriptors (masks of popcount 2..L-1), per-owner offsets padded to 4
  std::vector<DpDesc> desc;
  std::vector<uint32_t> offm(1u << L, 0);
  uint32_t ksz = 0;
  for (uint32_t d = 2; d < L; ++d) {
    pl->desc_begin[d] = (uint32_t)desc.size();
    for (uint32_t mask = 0; mask < (1u << L); ++mask) {
      if ((uint32_t)__builtin_popcount(mask) != d) continue;
      DpDesc ds{};
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
  for (uint32_t k = 0; k < L; ++k) {
    uint32_t src = ((1u << L) - 1) & ~(1u << k);
    pl->final_src[k] = (L - 1 == 1) ? (kURow | (uint32_t)__builtin_ctz(src)) : offm[src];
  }
  // final-level tiles: rows r (colex prefixes, order L-1), columns j
  std::vector<int2> tiles;
  const uint32_t *stL = &starts[(size_t)L * (R + 1)];
  for (uint32_t j0 = 0; j0 < pl->R4; j0 += 4) {
    uint32_t jl = std::min(j0 + 3, R - 1);
    uint32_t cnt = stL[jl + 1] - stL[jl];
    for (uint32_t r0 = 0; r0 < cnt; r0 += 4) tiles.push_back(make_int2((int)r0, (int)j0));
  }
  pl->ntiles = (uint32_t)tiles.size();
  if (pl->ntiles <= (uint32_t)kThreads) {
    pl->NT = 1;
    pl->G = std::max(1u, std::min(8u, (uint32_t)kThreads / pl->ntiles));
  } else {
    pl->G = 1;
    uint32_t nt = (pl->ntiles + kThreads - 1) / kThreads;
    int NT = 1;
    while ((uint32_t)NT < nt) NT *= 2;
    if (NT > 8) return pl;
    pl->NT = NT;
  }
  // colex -> lex permutation of the output
  std::vector<uint32_t> lex(pl->m[L]);
  for_each_sorted(R, (int)L, [&](const std::vector<uint32_t> &q, uint64_t lin) {
    uint64_t cx = 0;
    for (uint32_t i = 0; i < L; ++i) cx += symsize(q[i], i + 1);  // C(q_i + i, i + 1)
    lex[cx] = (uint32_t)lin;
  });
  // shared memory and batch size per precision
  for (int pi = 0; pi < 2; ++pi) {
    const size_t es = pi == 0 ? 8 : 4;
    size_t fixed = (((size_t)(L + 1) * (R + 1) * 4) + 15) / 16 * 16 + ((size_t)pl->jtab_len + 15) / 16 * 16 +
                   ((size_t)pl->ndesc * sizeof(DpDesc) + 15) / 16 * 16;
    size_t per_owner = (2 * (size_t)L * pl->R4 + pl->ksz4) * es;
    const size_t budget = 110 * 1024;
    if (fixed + per_owner > 220 * 1024) return pl;
    uint32_t bo = (uint32_t)std::min<size_t>(32, (budget > fixed ? (budget - fixed) / per_owner : 0));
    if (bo < 1) bo = 1;
    // the group reduction reuses the staging area
    size_t red = (size_t)(pl->G > 1 ? pl->G - 1 : 0) * pl->ntiles * 16 * es;
    size_t stage = (size_t)bo * (2 * (size_t)L * pl->R4 + pl->ksz4) * es;
    while (stage < red) { ++bo; stage = (size_t)bo * (2 * (size_t)L * pl->R4 + pl->ksz4) * es; }
    pl->BO[pi] = bo;
    pl->smem[pi] = fixed + stage;
    if (pl->smem[pi] > 227 * 1024) return pl;
  }
  pl->starts.alloc(starts.size());
  SPB_CUDA(cudaMemcpy(pl->starts.p, starts.data(), starts.size() * 4, cudaMemcpyHostToDevice));
  pl->jtab.alloc(std::max<size_t>(jt.size(), 1));
  if (!jt.empty()) SPB_CUDA(cudaMemcpy(pl->jtab.p, jt.data(), jt.size(), cudaMemcpyHostToDevice));
  pl->desc.alloc(std::max<size_t>(desc.size(), 1));
  if (!desc.empty())
    SPB_CUDA(cudaMemcpy(pl->desc.p, desc.data(), desc.size() * sizeof(DpDesc), cudaMemcpyHostToDevice));
  pl->tiles.alloc(tiles.size());
  SPB_CUDA(cudaMemcpy(pl->tiles.p, tiles.data(), tiles.size() * sizeof(int2), cudaMemcpyHostToDevice));
  pl->lexidx.alloc(lex.size());
  SPB_CUDA(cudaMemcpy(pl->lexidx.p, lex.data(), lex.size() * 4, cudaMemcpyHostToDevice));
  pl->ok = true;
  return pl;
}

bool tiled_supported(const TiledPlan &pl) { return pl.ok; }

template <int L, int NT, typename T>
static void launch_tiled_t(const TiledParams &tp, uint32_t nchunks, size_t smem, cudaStream_t st) {
  auto kern = s3ttmc_tiled_kernel<L, NT, T>;
  SPB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kern<<<nchunks, kThreads, smem, st>>>(tp);
  SPB_LAUNCH_CHECK();
}

template <int L, typename T>
static void launch_tiled_nt(int NT, const TiledParams &tp, uint32_t nchunks, size_t smem,
                            cudaStream_t st) {
  switch (NT) {
    case 1: launch_tiled_t<L, 1, T>(tp, nchunks, smem, st); break;
    case 2: launch_tiled_t<L, 2, T>(tp, nchunks, smem, st); break;
    case 4: launch_tiled_t<L, 4, T>(tp, nchunks, smem, st); break;
    default: launch_tiled_t<L, 8, T>(tp, nchunks, smem, st); break;
  }
}

template <typename T>
static void launch_tiled_l(uint32_t L, int NT, const TiledParams &tp, uint32_t nchunks, size_t smem,
                           cudaStream_t st) {
  switch (L) {
    case 2: launch_tiled_nt<2, T>(NT, tp, nchunks, smem, st); break;
    case 3: launch_tiled_nt<3, T>(NT, tp, nchunks, smem, st); break;
    case 4: launch_tiled_nt<4, T>(NT, tp, nchunks, smem, st); break;
    case 5: launch_tiled_nt<5, T>(NT, tp, nchunks, smem, st); break;
    case 6: launch_tiled_nt<6, T>(NT, tp, nchunks, smem, st); break;
    default: launch_tiled_nt<7, T>(NT, tp, nchunks, smem, st); break;
  }
}

void tiled_launch(const TiledPlan &pl, const TensorState &t, const ItemSet &items, const void *dU, void *dYpacked,
                  int precision, cudaStream_t st) {
  const int pi = precision == SYMPROP_FP64 ? 0 : 1;
  TiledParams tp{};
  tp.chunks = items.chunks;
  tp.own_S = t.own_S.p;
  tp.own_c = pi == 0 ? (const void *)t.own_c64.p : (const void *)t.own_c32.p;
  tp.sstride = t.sstride;
  tp.U = dU;
  tp.R = pl.R;
  tp.R4 = pl.R4;
  tp.Y = dYpacked;
  tp.ldy = pl.m[pl.L];
  tp.partials = t.partials.p;
  tp.mL = pl.m[pl.L];
  tp.starts = pl.starts.p;
  tp.jtab = pl.jtab.p;
  tp.jtab_len = pl.jtab_len;
  tp.desc = pl.desc.p;
  tp.ndesc = pl.ndesc;
  for (int d = 0; d <= kMaxLt; ++d) {
    tp.jtab_off[d] = pl.jtab_off[d];
    tp.desc_begin[d] = pl.desc_begin[d];
    tp.desc_count[d] = pl.desc_count[d];
    tp.m4[d] = pl.m4[d];
    tp.m[d] = pl.m[d];
  }
  for (int k = 0; k < kMaxLt; ++k) tp.final_src[k] = pl.final_src[k];
  tp.tiles = pl.tiles.p;
  tp.ntiles = pl.ntiles;
  tp.lexidx = pl.lexidx.p;
  tp.ksz4 = pl.ksz4;
  tp.BO = pl.BO[pi];
  tp.G = pl.G;
  tp.nown = t.nown;
  tp.nrows = t.dim;
  tp.nslots = t.nslots;
  if (!items.nchunks) return;
  if (pi == 0) launch_tiled_l<double>(pl.L, pl.NT, tp, items.nchunks, pl.smem[0], st);
  else launch_tiled_l<float>(pl.L, pl.NT, tp, items.nchunks, pl.smem[1], st);
  spb_check_host(st, "S3TTMc tiled kernel");
}

}  // namespace spb
