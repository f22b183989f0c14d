// S3TTMc on sm_100a: Y[i] = sum over owners (i, S, c) of c * K(S), where
// K(S) is the packed symmetric tensor of the (N-1)-multiset S built by the
// reference's level recursion K(S) = sum_k K(S \ s_k) (x) U[s_k]
// (SymOuterProd, include/detail/dense/symtensor.hpp:24-39, swept level by
// level in CompressedDTree::kronecker_product_opt5,
// src/compressed_dtree.cpp:421-518).
//
// B200 design (differs from opt5 on purpose):
//  * one CTA per work item = a row of Y, or a slice of a long row; owners are
//    pre-sorted by row, so Y is produced by a segmented reduction in
//    registers; rows cut into slices write FP64 partial rows that a second
//    kernel adds in a fixed order: no global atomics, deterministic;
//  * no tree level is materialised: the intermediate tensors K(P) of every
//    sub-multiset P of the leaf are recomputed per owner in shared memory
//    from U rows.  U (n x R) stays L2-resident (12.8 MB at n=200k, R=16),
//    so the HBM stream is the owner list in and Y out.  This removes the
//    level-(N-2) array that opt5 allocates (88 GB at 5M order-4 tuples);
//  * FP32 mode accumulates each owner's contribution in FP32 and folds
//    batches into a Kahan-compensated accumulator.
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>

#include "check.cuh"
#include "s3ttmc_chain.cuh"
#include "s3ttmc_tiled.cuh"
#include "s3ttmc_warp.cuh"
#include "tensor.cuh"

namespace spb {

static void finish_rows(TensorState &t, const ItemSet &items, uint64_t m, void *Ypk, bool packed, void *dY,
                        uint32_t R, uint32_t L, int precision, cudaStream_t st);

static constexpr int kMaxL = 7;          // orders 2..8
static constexpr uint32_t kURow = 0x80000000u;

struct MaskDesc {
  uint32_t dst;          // offset of this sub-multiset's tensor in sK
  uint32_t nterm;
  uint32_t src[kMaxL];   // sK offset, or kURow | position for a single id
  uint32_t k[kMaxL];     // position whose U row multiplies the term
};

struct PackedTables {
  uint32_t L = 0, R = 0;
  uint64_t m[kMaxL + 1] = {};
  // device: inner tables (levels 2..L-1) then the final level
  DBuf<uint32_t> tab;
  uint32_t tab_inner_len = 0;
  uint32_t tab_level_off[kMaxL + 1] = {};  // offsets into tab for levels 2..L
  DBuf<MaskDesc> desc;
  uint32_t ndesc = 0;
  uint32_t level_desc_begin[kMaxL + 1] = {}, level_desc_count[kMaxL + 1] = {};
  uint32_t final_src[kMaxL] = {};
  uint32_t ksize = 0;  // elements of sK
  int threads = 256, maxpt = 1;
  size_t smem_bytes[2] = {0, 0};  // by precision
};

// ---------------------------------------------------------------- tables

static std::shared_ptr<PackedTables> build_tables(uint32_t N, uint32_t R) {
  auto tb = std::make_shared<PackedTables>();
  const uint32_t L = N - 1;
  tb->L = L;
  tb->R = R;
  for (uint32_t d = 0; d <= L; ++d) tb->m[d] = symsize(R, d);
  if (R > 255) fail(SYMPROP_ERR_SIZE, "rank %u > 255 not supported", R);
  // packed recursion tables: entry q of level d -> (prefix index << 8) | last
  std::vector<uint32_t> tab;
  for (uint32_t d = 2; d <= L; ++d) {
    if (tb->m[d - 1] >= (1ull << 24)) fail(SYMPROP_ERR_SIZE, "packed size too large");
    tb->tab_level_off[d] = (uint32_t)tab.size();
    // prefix index = linear index of q[0..d-2] in level d-1 enumeration
    std::vector<uint32_t> q_prev;
    uint64_t prev_lin = 0;
    // enumerate level d; prefix changes exactly when q[0..d-2] changes, and
    // prefixes appear in level d-1 order, so a running counter suffices
    std::vector<uint32_t> last_prefix;
    bool first = true;
    for_each_sorted(R, (int)d, [&](const std::vector<uint32_t> &q, uint64_t) {
      std::vector<uint32_t> pre(q.begin(), q.end() - 1);
      if (!first && pre != last_prefix) ++prev_lin;
      first = false;
      last_prefix = pre;
      tab.push_back((uint32_t)(prev_lin << 8) | q.back());
    });
    (void)q_prev;
  }
  tb->tab_inner_len = L >= 3 ? tb->tab_level_off[L] : 0;
  if (L < 2) tb->tab_level_off[L] = 0;
  // DP over position subsets of the leaf, popcount 2..L-1
  std::vector<MaskDesc> desc;
  std::vector<uint32_t> off_of_mask(1u << L, 0);
  uint32_t ksz = 0;
  for (uint32_t d = 2; d + 1 <= L; ++d) {
    tb->level_desc_begin[d] = (uint32_t)desc.size();
    for (uint32_t mask = 0; mask < (1u << L); ++mask) {
      if ((uint32_t)__builtin_popcount(mask) != d) continue;
      MaskDesc md{};
      md.dst = ksz;
      off_of_mask[mask] = ksz;
      ksz += (uint32_t)tb->m[d];
      md.nterm = 0;
      for (uint32_t k = 0; k < L; ++k) {
        if (!(mask & (1u << k))) continue;
        uint32_t src = mask & ~(1u << k);
        md.src[md.nterm] = (d - 1 == 1) ? (kURow | (uint32_t)__builtin_ctz(src)) : off_of_mask[src];
        md.k[md.nterm] = k;
        md.nterm++;
      }
      desc.push_back(md);
    }
    tb->level_desc_count[d] = (uint32_t)desc.size() - tb->level_desc_begin[d];
  }
  for (uint32_t k = 0; k < L; ++k) {
    uint32_t src = ((1u << L) - 1) & ~(1u << k);
    tb->final_src[k] = (L - 1 == 1) ? (kURow | (uint32_t)__builtin_ctz(src))
                       : (L - 1 == 0) ? kURow : off_of_mask[src];
  }
  tb->ksize = ksz;
  tb->ndesc = (uint32_t)desc.size();
  tb->tab.alloc(std::max<size_t>(tab.size(), 1));
  if (!tab.empty())
    SPB_CUDA(cudaMemcpy(tb->tab.p, tab.data(), tab.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
  tb->desc.alloc(std::max<size_t>(desc.size(), 1));
  if (!desc.empty())
    SPB_CUDA(cudaMemcpy(tb->desc.p, desc.data(), desc.size() * sizeof(MaskDesc), cudaMemcpyHostToDevice));
  // launch shape
  const uint64_t mL = tb->m[L];
  const int threads = 256;
  uint64_t per = (mL + threads - 1) / threads;
  if (per > 64) fail(SYMPROP_ERR_SIZE, "packed output width %llu too large", (unsigned long long)mL);
  int maxpt = 1;
  while ((uint64_t)maxpt < per) maxpt *= 2;
  tb->threads = threads;
  tb->maxpt = maxpt;
  for (int p = 0; p < 2; ++p) {
    size_t es = p == 0 ? sizeof(double) : sizeof(float);
    size_t b = 0;
    b += (size_t)tb->tab_inner_len * 4;
    b = (b + 15) / 16 * 16;
    b += (size_t)tb->ndesc * sizeof(MaskDesc);
    b = (b + 15) / 16 * 16;
    b += 2 * (size_t)L * R * es;
    b = (b + 15) / 16 * 16;
    b += (size_t)ksz * es;
    tb->smem_bytes[p] = b;
  }
  return tb;
}

// --------------------------------------------------------------- kernels

struct RowParams {
  const Chunk *chunks;
  const uint32_t *own_S;
  const void *own_c;
  uint32_t sstride;
  const void *U;
  uint32_t R;
  void *Y;           // dim x ldy (T), packed
  uint64_t ldy;
  double *partials;  // nslots x mL
  const uint32_t *tab;
  uint32_t tab_inner_len;
  uint32_t tab_final_off;
  const MaskDesc *desc;
  uint32_t ndesc;
  uint32_t ksize;
  uint32_t mlev[kMaxL + 1];
  uint32_t tab_off[kMaxL + 1];
  uint32_t desc_begin[kMaxL + 1];
  uint32_t desc_count[kMaxL + 1];
  uint32_t final_src[kMaxL];
  uint64_t nown;  // bounds the checked build tests
  uint32_t nrows, nslots;
};

template <typename T> struct Acc;
template <> struct Acc<double> {
  static constexpr int kBatch = 1 << 30;
};
template <> struct Acc<float> {
  static constexpr int kBatch = 8;  // owners summed plainly before a compensated fold
};

template <int L, int MAXPT, typename T>
__global__ void __launch_bounds__(256, 1) s3ttmc_rows_kernel(const RowParams p) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int tid = threadIdx.x, nt = blockDim.x;
  const Chunk ch = p.chunks[blockIdx.x];
  if (!SPB_BOUND(ch.ob <= ch.oe && ch.oe <= p.nown && ch.row < p.nrows && (ch.slot == kDirect || ch.slot < p.nslots),
                 301, blockIdx.x))
    return;  // the whole CTA leaves (the chunk is the CTA's)
  const uint32_t R = p.R;

  uint32_t *sTab = reinterpret_cast<uint32_t *>(smem);
  size_t off = ((size_t)p.tab_inner_len * 4 + 15) / 16 * 16;
  MaskDesc *sDesc = reinterpret_cast<MaskDesc *>(smem + off);
  off += ((size_t)p.ndesc * sizeof(MaskDesc) + 15) / 16 * 16;
  T *sU = reinterpret_cast<T *>(smem + off);
  T *sW = sU + L * R;
  off += ((size_t)2 * L * R * sizeof(T) + 15) / 16 * 16;
  T *sK = reinterpret_cast<T *>(smem + off);

  for (uint32_t i = tid; i < p.tab_inner_len; i += nt) sTab[i] = p.tab[i];
  {
    const uint32_t *src = reinterpret_cast<const uint32_t *>(p.desc);
    uint32_t *dst = reinterpret_cast<uint32_t *>(sDesc);
    const uint32_t words = p.ndesc * (uint32_t)(sizeof(MaskDesc) / 4);
    for (uint32_t i = tid; i < words; i += nt) dst[i] = src[i];
  }

  constexpr bool kExact = sizeof(T) == 8;  // FP64 accumulates directly
  const uint32_t mL = p.mlev[L];
  uint32_t ftab[MAXPT];
#pragma unroll
  for (int j = 0; j < MAXPT; ++j) {
    uint32_t q = tid + j * nt;
    ftab[j] = q < mL ? p.tab[p.tab_final_off + q] : 0u;
  }
  T acc[MAXPT], cmp[MAXPT], tmp[MAXPT];
#pragma unroll
  for (int j = 0; j < MAXPT; ++j) { acc[j] = T(0); cmp[j] = T(0); tmp[j] = T(0); }

  const T *U = reinterpret_cast<const T *>(p.U);
  const T *own_c = reinterpret_cast<const T *>(p.own_c);
  int batch = 0;
  __syncthreads();

  for (uint64_t o = ch.ob; o < ch.oe; ++o) {
    // stage the leaf's U rows, and the coefficient-scaled copy for the last level
    const uint32_t *S = p.own_S + o * p.sstride;
    const T c = own_c[o];
    for (uint32_t i = tid; i < L * R; i += nt) {
      uint32_t k = i / R, x = i - k * R;
      const uint32_t id = S[k];
      T u = SPB_BOUND(id < p.nrows, 302, id) ? U[(uint64_t)id * R + x] : T(0);
      sU[i] = u;
      sW[i] = c * u;
    }
    __syncthreads();
    // intermediate sub-multiset tensors, level by level
#pragma unroll 1
    for (int d = 2; d < L; ++d) {
      const uint32_t md = p.mlev[d];
      const uint32_t items = p.desc_count[d] * md;
      const uint32_t *tabd = sTab + p.tab_off[d];
      for (uint32_t it = tid; it < items; it += nt) {
        uint32_t mi = it / md, q = it - mi * md;
        const MaskDesc &ds = sDesc[p.desc_begin[d] + mi];
        uint32_t e = tabd[q];
        uint32_t pre = e >> 8, last = e & 0xffu;
        T v = T(0);
        for (uint32_t t = 0; t < ds.nterm; ++t) {
          uint32_t s = ds.src[t];
          T a = (s & kURow) ? sU[(s & 0xffu) * R + pre] : sK[s + pre];
          v += a * sU[ds.k[t] * R + last];
        }
        sK[ds.dst + q] = v;
      }
      __syncthreads();
    }
    // last level: contribution c*K(S) for this thread's outputs
#pragma unroll
    for (int j = 0; j < MAXPT; ++j) {
      uint32_t q = tid + j * nt;
      if (q < mL) {
        uint32_t pre = ftab[j] >> 8, last = ftab[j] & 0xffu;
        T v = T(0);
#pragma unroll
        for (int k = 0; k < L; ++k) {
          uint32_t s = p.final_src[k];
          T a = (s & kURow) ? sU[(s & 0xffu) * R + pre] : sK[s + pre];
          v += a * sW[k * R + last];
        }
        if constexpr (kExact) acc[j] += v; else tmp[j] += v;
      }
    }
    if (!kExact && ++batch >= Acc<T>::kBatch) {
#pragma unroll
      for (int j = 0; j < MAXPT; ++j) {  // Kahan fold of the batch
        T y = tmp[j] - cmp[j];
        T s = acc[j] + y;
        cmp[j] = (s - acc[j]) - y;
        acc[j] = s;
        tmp[j] = T(0);
      }
      batch = 0;
    }
    __syncthreads();
  }
  if constexpr (!kExact) {
#pragma unroll
    for (int j = 0; j < MAXPT; ++j) {
      T y = tmp[j] - cmp[j];
      T s = acc[j] + y;
      cmp[j] = (s - acc[j]) - y;
      acc[j] = s;
    }
  }
  if (ch.slot == kDirect) {
    T *Y = reinterpret_cast<T *>(p.Y) + (uint64_t)ch.row * p.ldy;
#pragma unroll
    for (int j = 0; j < MAXPT; ++j) {
      uint32_t q = tid + j * nt;
      if (q < mL) Y[q] = acc[j] - cmp[j];
    }
  } else {
    double *P = p.partials + (uint64_t)ch.slot * mL;
#pragma unroll
    for (int j = 0; j < MAXPT; ++j) {
      uint32_t q = tid + j * nt;
      if (q < mL) P[q] = (double)acc[j] - (double)cmp[j];
    }
  }
}

// rows cut into slices: add the FP64 partials in slot order
// grid (split rows, column blocks of 32): warp w adds slots w, w+8, ... for
// 32 consecutive columns (coalesced), then the 8 warp sums are added in
// warp order (deterministic)
template <typename T>
__global__ void __launch_bounds__(256) combine_kernel(const SplitRow *split, const double *partials,
                                                      uint32_t mL, void *Yv, uint64_t ldy, uint32_t nrows,
                                                      uint32_t nslots) {
  __shared__ double red[8][32];
  const SplitRow s = split[blockIdx.x];
  if (!SPB_BOUND(s.row < nrows && s.slot_begin <= s.slot_end && s.slot_end <= nslots, 401, blockIdx.x))
    return;  // the whole CTA leaves (the split row is the CTA's)
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t q = blockIdx.y * 32 + lane;
  double a = 0.0;
  if (q < mL)
    for (uint32_t k = s.slot_begin + warp; k < s.slot_end; k += 8) a += partials[(uint64_t)k * mL + q];
  red[warp][lane] = a;
  __syncthreads();
  if (warp == 0 && q < mL) {
    double t = 0.0;
#pragma unroll
    for (int w = 0; w < 8; ++w) t += red[w][lane];
    reinterpret_cast<T *>(Yv)[(uint64_t)s.row * ldy + q] = (T)t;
  }
}

// unpack packed order-`order` rows into dim^order full rows
// (SymtensorOps::ToTensor, include/detail/dense/symtensor.hpp:96-116)
template <typename T>
__global__ void unpack_kernel(const T *packed, uint64_t rows, uint64_t m, uint32_t dim,
                              uint32_t order, uint64_t full_cols, T *full) {
  uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= rows * full_cols) return;
  uint64_t r = idx / full_cols, f = idx - r * full_cols;
  uint32_t q[16];
  uint64_t x = f;
  for (int j = (int)order - 1; j >= 0; --j) {
    q[j] = (uint32_t)(x % dim);
    x /= dim;
  }
  for (uint32_t a = 1; a < order; ++a) {  // sort
    uint32_t v = q[a];
    int b = (int)a - 1;
    while (b >= 0 && q[b] > v) { q[b + 1] = q[b]; --b; }
    q[b + 1] = v;
  }
  // packed offset (SymtensorOps::At, symtensor.hpp:83-94) via binomials
  uint64_t pos = 0;
  uint32_t start = 0;
  for (uint32_t j = 0; j < order; ++j) {
    uint32_t rem = order - 1 - j;
    for (uint32_t i = start; i < q[j]; ++i) {
      // symsize(dim - i, rem) = C(dim - i + rem - 1, rem)
      uint64_t n = (uint64_t)(dim - i) + rem - 1, k = rem, c = 1;
      if (k > n) c = 0;
      else {
        if (2 * k > n) k = n - k;
        for (uint64_t t = 1; t <= k; ++t) c = c * (n - k + t) / t;
      }
      pos += c;
    }
    start = q[j];
  }
  if (!SPB_BOUND(order <= 16 && pos < m, 402, pos)) return;
  full[idx] = packed[r * m + pos];
}

// --------------------------------------------------------------- launch

template <int L, typename T>
static void launch_rows(const PackedTables &tb, const RowParams &rp, uint32_t nchunks,
                        size_t smem, cudaStream_t st) {
  auto go = [&](auto kern) {
    if (smem > 48 * 1024)
      SPB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<nchunks, tb.threads, smem, st>>>(rp);
    SPB_LAUNCH_CHECK();
  };
  switch (tb.maxpt) {
    case 1: go(s3ttmc_rows_kernel<L, 1, T>); break;
    case 2: go(s3ttmc_rows_kernel<L, 2, T>); break;
    case 4: go(s3ttmc_rows_kernel<L, 4, T>); break;
    case 8: go(s3ttmc_rows_kernel<L, 8, T>); break;
    case 16: go(s3ttmc_rows_kernel<L, 16, T>); break;
    case 32: go(s3ttmc_rows_kernel<L, 32, T>); break;
    default: go(s3ttmc_rows_kernel<L, 64, T>); break;
  }
}

template <typename T>
static void dispatch_rows(uint32_t L, const PackedTables &tb, const RowParams &rp,
                          uint32_t nchunks, size_t smem, cudaStream_t st) {
  switch (L) {
    case 2: launch_rows<2, T>(tb, rp, nchunks, smem, st); break;
    case 3: launch_rows<3, T>(tb, rp, nchunks, smem, st); break;
    case 4: launch_rows<4, T>(tb, rp, nchunks, smem, st); break;
    case 5: launch_rows<5, T>(tb, rp, nchunks, smem, st); break;
    case 6: launch_rows<6, T>(tb, rp, nchunks, smem, st); break;
    case 7: launch_rows<7, T>(tb, rp, nchunks, smem, st); break;
    default: fail(SYMPROP_ERR_ORDER, "order %u not supported by S3TTMc", L + 1);
  }
}

static PackedTables &tables_for(TensorState &t, uint32_t R) {
  auto it = t.tables.find(R);
  if (it != t.tables.end()) return *it->second;
  auto tb = build_tables(t.order, R);
  auto &ref = *tb;
  t.tables[R] = tb;
  return ref;
}

uint32_t s3ttmc_launch_count(const TensorState &t, uint32_t R, bool packed) {
  if (t.order <= 2) return packed ? 1 : 1;
  const bool chain = (s3ttmc_schedule() == kScheduleAuto || s3ttmc_schedule() == kScheduleChain) &&
                     chain_supported(t, R);
  const uint32_t nsplit = chain && t.chain ? t.chain->nsplit : t.nsplit;
  uint32_t n = 1;                 // S3TTMc kernel
  if (chain && t.chain && t.chain->nlight) n += 1;  // warp kernel of the light rows
  if (nsplit) n += 1;             // combine kernel
  if (!packed) n += 1;            // unpack kernel
  return n;
}

void unpack_rows(const void *dpacked, uint64_t rows, uint32_t dim, uint32_t order, void *dfull,
                 int precision, cudaStream_t st) {
  uint64_t m = symsize(dim, order);
  uint64_t full = 1;
  for (uint32_t j = 0; j < order; ++j) full *= dim;
  uint64_t total = rows * full;
  if (!total) return;
  unsigned grid = (unsigned)((total + 255) / 256);
  if (precision == SYMPROP_FP64)
    unpack_kernel<double><<<grid, 256, 0, st>>>((const double *)dpacked, rows, m, dim, order, full,
                                                (double *)dfull);
  else
    unpack_kernel<float><<<grid, 256, 0, st>>>((const float *)dpacked, rows, m, dim, order, full,
                                               (float *)dfull);
  SPB_LAUNCH_CHECK();
  spb_check_host(st, "unpack");
}

// A second stream of this device (created once, kept), forked from `st`
// at construction: work queued on `side` starts after the work queued on
// `st` so far, and join() makes later work on `st` wait for it.
struct SideFork {
  cudaStream_t st, side;
  cudaEvent_t forked = nullptr, done = nullptr;
  bool joined = false;
  explicit SideFork(cudaStream_t s) : st(s) {
    static std::mutex mu;
    static std::map<int, cudaStream_t> sides;
    int dev = 0;
    SPB_CUDA(cudaGetDevice(&dev));
    {
      std::lock_guard<std::mutex> lock(mu);
      auto it = sides.find(dev);
      if (it == sides.end()) {
        cudaStream_t x;
        SPB_CUDA(cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking));
        it = sides.emplace(dev, x).first;
      }
      side = it->second;
    }
    SPB_CUDA(cudaEventCreateWithFlags(&forked, cudaEventDisableTiming));
    SPB_CUDA(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
    SPB_CUDA(cudaEventRecord(forked, st));
    SPB_CUDA(cudaStreamWaitEvent(side, forked, 0));
  }
  void join() {
    SPB_CUDA(cudaEventRecord(done, side));
    SPB_CUDA(cudaStreamWaitEvent(st, done, 0));
    joined = true;
  }
  ~SideFork() {
    if (!joined) {  // an exception between fork and join: still order the streams
      cudaEventRecord(done, side);
      cudaStreamWaitEvent(st, done, 0);
    }
    cudaEventDestroy(forked);
    cudaEventDestroy(done);
  }
};

// One pass over a set of work items: writes the packed rows (or, when
// `packed` is false, the full rows) [items.row0, items.row0 + items.rows) of
// dY.  t.partials and t.scratch must already be large enough.
static void s3ttmc_items(TensorState &t, const ItemSet &items, const void *dU, uint32_t R, bool packed,
                         void *dY, int precision, cudaStream_t st) {
  const size_t es = precision == SYMPROP_FP64 ? 8 : 4;
  const uint32_t L = t.order - 1;
  const uint64_t m = symsize(R, L);
  uint64_t full = 1;
  for (uint32_t j = 0; j < L; ++j) full *= R;
  const uint64_t ldy = packed ? m : full;
  if (t.order == 2) {
    // The reference's level loop is empty for depth 1 and Y stays zero
    // (src/compressed_dtree.cpp:451).
    if (items.rows)
      SPB_CUDA(cudaMemsetAsync((char *)dY + (size_t)items.row0 * ldy * es, 0, (size_t)items.rows * ldy * es, st));
    return;
  }
  void *Ypk = packed ? dY : (void *)t.scratch.p;
  const int sched = s3ttmc_schedule();
  if (items.chain) {
    // light rows on the warp-per-row kernel (the chain kernel where that
    // kernel does not cover R), heavy rows on the chain kernel
    if (items.nlight) {
      ItemSet light;
      light.chunks = items.light;
      light.nchunks = items.nlight;
      light.row0 = items.row0;
      light.rows = items.rows;
      auto it = t.warp.find(R);
      if (it == t.warp.end()) it = t.warp.emplace(R, warp_plan(t.order, R)).first;
      if (warp_supported(*it->second)) {
        // the two kernels write disjoint rows: the light rows run on a side
        // stream, forked from and joined back into `st`, beside the chain
        // kernel (which leaves most issue slots idle)
        SideFork fork(st);
        warp_launch(*it->second, t, light, dU, Ypk, precision, fork.side);
        chain_launch(t, *t.chain, items, dU, R, Ypk, precision, st);
        fork.join();
      } else {
        light.chain = true;
        chain_launch(t, *t.chain, light, dU, R, Ypk, precision, st);
        chain_launch(t, *t.chain, items, dU, R, Ypk, precision, st);
      }
    } else {
      chain_launch(t, *t.chain, items, dU, R, Ypk, precision, st);
    }
    finish_rows(t, items, m, Ypk, packed, dY, R, L, precision, st);
    return;
  }
  if (sched == kScheduleAuto || sched == kScheduleWarp) {
    auto it = t.warp.find(R);
    if (it == t.warp.end()) it = t.warp.emplace(R, warp_plan(t.order, R)).first;
    if (warp_supported(*it->second)) {
      warp_launch(*it->second, t, items, dU, Ypk, precision, st);
      finish_rows(t, items, m, Ypk, packed, dY, R, L, precision, st);
      return;
    }
    if (sched == kScheduleWarp)
      fail(SYMPROP_ERR_SIZE, "warp S3TTMc does not support order %u rank %u", t.order, R);
  }
  if (sched == kScheduleAuto || sched == kScheduleTiled) {
    auto it = t.tiled.find(R);
    if (it == t.tiled.end()) it = t.tiled.emplace(R, tiled_plan(t.order, R)).first;
    if (tiled_supported(*it->second)) {
      tiled_launch(*it->second, t, items, dU, Ypk, precision, st);
      finish_rows(t, items, m, Ypk, packed, dY, R, L, precision, st);
      return;
    }
    if (sched == kScheduleTiled)
      fail(SYMPROP_ERR_SIZE, "tiled S3TTMc does not support order %u rank %u", t.order, R);
  }
  PackedTables &tb = tables_for(t, R);

  RowParams rp{};
  rp.chunks = items.chunks;
  rp.own_S = t.own_S.p;
  rp.own_c = precision == SYMPROP_FP64 ? (const void *)t.own_c64.p : (const void *)t.own_c32.p;
  rp.sstride = t.sstride;
  rp.U = dU;
  rp.R = R;
  rp.Y = Ypk;
  rp.ldy = m;
  rp.partials = t.partials.p;
  rp.tab = tb.tab.p;
  rp.tab_inner_len = tb.tab_inner_len;
  rp.tab_final_off = tb.tab_level_off[L];
  rp.desc = tb.desc.p;
  rp.ndesc = tb.ndesc;
  rp.ksize = tb.ksize;
  for (uint32_t d = 0; d <= L && d <= (uint32_t)kMaxL; ++d) {
    rp.mlev[d] = (uint32_t)tb.m[d];
    rp.tab_off[d] = tb.tab_level_off[d];
    rp.desc_begin[d] = tb.level_desc_begin[d];
    rp.desc_count[d] = tb.level_desc_count[d];
  }
  for (uint32_t k = 0; k < L; ++k) rp.final_src[k] = tb.final_src[k];
  rp.nown = t.nown;
  rp.nrows = t.dim;
  rp.nslots = t.nslots;
  const size_t smem = tb.smem_bytes[precision == SYMPROP_FP64 ? 0 : 1];
  if (smem > 227 * 1024)
    fail(SYMPROP_ERR_SIZE, "order %u rank %u needs %zu bytes of shared memory", t.order, R, smem);
  if (items.nchunks) {
    if (precision == SYMPROP_FP64)
      dispatch_rows<double>(L, tb, rp, items.nchunks, smem, st);
    else
      dispatch_rows<float>(L, tb, rp, items.nchunks, smem, st);
    spb_check_host(st, "S3TTMc rows kernel");
  }
  finish_rows(t, items, m, Ypk, packed, dY, R, L, precision, st);
}

// make room for the partial sums of split rows and, for full output, the
// packed staging rows
// whether this call runs the pivot-chain schedule
static bool use_chain(const TensorState &t, uint32_t R) {
  const int sched = s3ttmc_schedule();
  if (sched == kScheduleChain && !chain_supported(t, R))
    fail(SYMPROP_ERR_SIZE, "chain S3TTMc does not support order %u rank %u", t.order, R);
  return (sched == kScheduleAuto || sched == kScheduleChain) && chain_supported(t, R);
}

static void s3ttmc_reserve(TensorState &t, uint32_t R, bool packed, int precision) {
  if (R == 0) fail(SYMPROP_ERR_INVALID, "R must be positive");
  if (precision != SYMPROP_FP64 && precision != SYMPROP_FP32)
    fail(SYMPROP_ERR_INVALID, "unknown precision %d", precision);
  const size_t es = precision == SYMPROP_FP64 ? 8 : 4;
  const uint64_t m = symsize(R, t.order - 1);
  if (!packed && t.order > 2) t.scratch.ensure((size_t)t.dim * m * es);
  uint32_t slots = t.nslots;
  if (use_chain(t, R)) slots = std::max(slots, chain_data(t).nslots);
  if (slots) t.partials.ensure((size_t)slots * m);
}

void s3ttmc_prepare(TensorState &t, uint32_t R, bool packed, int precision) {
  s3ttmc_reserve(t, R, packed, precision);
}

void s3ttmc_run(TensorState &t, const void *dU, uint32_t R, bool packed, void *dY, int precision,
                cudaStream_t st) {
  NvtxRange nv("S3TTMc");
  s3ttmc_reserve(t, R, packed, precision);
  ItemSet all;
  if (use_chain(t, R)) {
    const ChainData &cd = chain_data(t);
    all.chunks = cd.chunks.p;
    all.nchunks = cd.nchunks;
    all.split = cd.split.p;
    all.nsplit = cd.nsplit;
    all.chain = true;
    all.nslots = cd.nslots;
    all.light = cd.light.p;
    all.nlight = cd.nlight;
  } else {
    all.chunks = t.chunks.p;
    all.nchunks = t.nchunks;
    all.split = t.split.p;
    all.nsplit = t.nsplit;
    all.nslots = t.nslots;
  }
  all.row0 = 0;
  all.rows = t.dim;
  s3ttmc_items(t, all, dU, R, packed, dY, precision, st);
}

// The compute and copy streams of the host-pointer call: created once per
// device, one right after the other, and kept for the life of the process.
static void host_streams(cudaStream_t &st, cudaStream_t &cp) {
  static std::mutex mu;
  static std::map<int, std::pair<cudaStream_t, cudaStream_t>> streams;
  int dev = 0;
  SPB_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  auto it = streams.find(dev);
  if (it == streams.end()) {
    cudaStream_t a, b;
    SPB_CUDA(cudaStreamCreateWithFlags(&a, cudaStreamNonBlocking));
    SPB_CUDA(cudaStreamCreateWithFlags(&b, cudaStreamNonBlocking));
    it = streams.emplace(dev, std::make_pair(a, b)).first;
  }
  st = it->second.first;
  cp = it->second.second;
}

// Number of row bands of the host-pointer call: one per 40 MiB of Y (about
// 0.75 ms of PCIe copy), at most 64 (SPB_HOST_BANDS overrides; one band = no
// overlap).  Each band costs a kernel tail; the last band's copy is not
// hidden.  On B200 over PCIe 5 the order-4 R=16 call (Y = 653 MB FP64) took
// 26.4 ms with 1 band, 16.8 with 8, 16.4 with 16 and 17.7 with 32 (compute
// alone 14.7 ms, copy alone 12 ms); an order-5 call with Y = 1.55 GB was
// flat (116.2-116.5 ms) from 16 to 48 bands.
static uint32_t host_band_count(size_t ybytes) {
  if (const char *e = std::getenv("SPB_HOST_BANDS")) {
    const long v = std::strtol(e, nullptr, 10);
    if (v >= 1) return (uint32_t)std::min<long>(v, 64);
  }
  const size_t per = 40ull << 20;
  return (uint32_t)std::max<size_t>(1, std::min<size_t>(64, (ybytes + per - 1) / per));
}

void s3ttmc_host(TensorState &t, const void *U, uint32_t R, bool packed, void *Y, int precision) {
  NvtxRange nv("S3TTMc (host buffers, row bands)");
  s3ttmc_reserve(t, R, packed, precision);
  const size_t es = precision == SYMPROP_FP64 ? 8 : 4;
  uint64_t cols = packed ? symsize(R, t.order - 1) : 1;
  if (!packed)
    for (uint32_t j = 0; j + 1 < t.order; ++j) cols *= R;
  const size_t ubytes = (size_t)t.dim * R * es, ybytes = (size_t)t.dim * cols * es;
  t.io_U.ensure(ubytes);
  t.io_Y.ensure(ybytes);
  const bool chain = use_chain(t, R);
  const RowBands &bd = chain ? chain_bands(t, host_band_count(ybytes)) : row_bands(t, host_band_count(ybytes));

  // SPB_TRACE_HOST=1 prints when each band's compute and copy ended
  const bool trace = std::getenv("SPB_TRACE_HOST") != nullptr;
  // compute on `st`, copy the finished bands back on `cp`; the guard waits
  // for both streams before the events go, also when a launch throws
  struct Events {
    cudaStream_t st = nullptr, cp = nullptr;
    std::vector<cudaEvent_t> done, copied;
    ~Events() {
      cudaStreamSynchronize(st);
      cudaStreamSynchronize(cp);
      for (cudaEvent_t e : done) cudaEventDestroy(e);
      for (cudaEvent_t e : copied) cudaEventDestroy(e);
    }
  } ss;
  host_streams(ss.st, ss.cp);
  const uint32_t nev = bd.nb + (trace ? 1 : 0);
  for (uint32_t k = 0; k < nev; ++k) {
    cudaEvent_t e;
    SPB_CUDA(cudaEventCreateWithFlags(&e, trace ? cudaEventDefault : cudaEventDisableTiming));
    ss.done.push_back(e);
    if (trace) {
      SPB_CUDA(cudaEventCreate(&e));
      ss.copied.push_back(e);
    }
  }
  if (trace) SPB_CUDA(cudaEventRecord(ss.done[bd.nb], ss.st));
  SPB_CUDA(cudaMemcpyAsync(t.io_U.p, U, ubytes, cudaMemcpyHostToDevice, ss.st));
  for (uint32_t k = 0; k < bd.nb; ++k) {
    ItemSet band;
    band.chunks = bd.chunks.p + bd.chunk0[k];
    band.nchunks = bd.chunk0[k + 1] - bd.chunk0[k];
    band.split = bd.split.p + bd.split0[k];
    band.nsplit = bd.split0[k + 1] - bd.split0[k];
    band.row0 = bd.row0[k];
    band.rows = bd.row0[k + 1] - bd.row0[k];
    band.chain = chain;
    band.nslots = chain ? t.chain->nslots : t.nslots;
    if (chain) {
      band.light = bd.light.p + bd.light0[k];
      band.nlight = bd.light0[k + 1] - bd.light0[k];
    }
    s3ttmc_items(t, band, t.io_U.p, R, packed, t.io_Y.p, precision, ss.st);
    SPB_CUDA(cudaEventRecord(ss.done[k], ss.st));
  }
  // all compute is queued before the first copy, so a copy into pageable
  // memory (which returns only when done) does not hold back the kernels
  for (uint32_t k = 0; k < bd.nb; ++k) {
    const size_t off = (size_t)bd.row0[k] * cols * es, len = (size_t)(bd.row0[k + 1] - bd.row0[k]) * cols * es;
    SPB_CUDA(cudaStreamWaitEvent(ss.cp, ss.done[k], 0));
    if (len) SPB_CUDA(cudaMemcpyAsync((char *)Y + off, t.io_Y.p + off, len, cudaMemcpyDeviceToHost, ss.cp));
    if (trace) SPB_CUDA(cudaEventRecord(ss.copied[k], ss.cp));
  }
  SPB_CUDA(cudaStreamSynchronize(ss.cp));
  SPB_CUDA(cudaStreamSynchronize(ss.st));
  if (trace)
    for (uint32_t k = 0; k < bd.nb; ++k) {
      float a = 0.f, b = 0.f;
      SPB_CUDA(cudaEventElapsedTime(&a, ss.done[bd.nb], ss.done[k]));
      SPB_CUDA(cudaEventElapsedTime(&b, ss.done[bd.nb], ss.copied[k]));
      std::fprintf(stderr, "[s3ttmc host] band %u/%u rows %u..%u items %u: computed %.3f ms, copied %.3f ms\n", k,
                   bd.nb, bd.row0[k], bd.row0[k + 1], bd.chunk0[k + 1] - bd.chunk0[k], a, b);
    }
  SPB_CUDA(cudaGetLastError());
}

// combine the partial rows of the set's split rows; unpack its rows if
// requested
static void finish_rows(TensorState &t, const ItemSet &items, uint64_t m, void *Ypk, bool packed, void *dY,
                        uint32_t R, uint32_t L, int precision, cudaStream_t st) {
  if (items.nsplit) {
    dim3 grid(items.nsplit, (unsigned)((m + 31) / 32));
    if (precision == SYMPROP_FP64)
      combine_kernel<double><<<grid, 256, 0, st>>>(items.split, t.partials.p, (uint32_t)m, Ypk, m, t.dim,
                                                   items.nslots);
    else
      combine_kernel<float><<<grid, 256, 0, st>>>(items.split, t.partials.p, (uint32_t)m, Ypk, m, t.dim,
                                                  items.nslots);
    SPB_LAUNCH_CHECK();
  }
  if (!packed && items.rows) {
    uint64_t full = 1;
    for (uint32_t j = 0; j < L; ++j) full *= R;
    const size_t es = precision == SYMPROP_FP64 ? 8 : 4;
    unpack_rows((const char *)Ypk + (size_t)items.row0 * m * es, items.rows, R, L,
                (char *)dY + (size_t)items.row0 * full * es, precision, st);
  }
  spb_check_host(st, "S3TTMc combine / unpack");
}

static std::atomic<int> g_schedule{kScheduleAuto};
int s3ttmc_schedule() { return g_schedule.load(); }
void set_s3ttmc_schedule(int s) { g_schedule.store(s); }

}  // namespace spb
