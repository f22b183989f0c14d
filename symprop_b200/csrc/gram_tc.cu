// The mixed-precision dense products of HOOI / HOQRI on the 5th-generation
// tensor cores (tcgen05): split-BF16 operands, FP32 accumulation in TMEM.
//
// The reference forms these products in FP64 with BLAS/LAPACK:
//   leftsvd(Y) (dgesvd)   src/sparse/spsymtensor.cpp:225, src/dense/matrixops.cpp:18-43
//   symsyrk  (Y D Y^T)    src/dense/matrixops.cpp:126-146 (AltHOOI)
//   symgemm  (Y D C^T)    src/dense/matrixops.cpp:102-124 (HOQRI)
// Here HOOI's leftsvd is the top eigenspace of the packed Gram (tucker.cu),
// and every product reads Z = Y D^1/2 (FP32, n x m) split once as Z ~ H + L,
// H = bf16(Z), L = bf16(Z - H), both row-major n x ld (ld = m rounded up to
// 64, zero padded).  A product of two split operands keeps three terms,
//     A B^T ~ Ah Bh^T + Ah Bl^T + Al Bh^T
// (the Al Bl^T term is about 2^-18 of the product and is dropped).
//
//   gram_cols  G = Z^T Z (m x m): both operands MN-major views of H / L
//              (a 64-wide column strip of Z is one 128-byte swizzled row per
//              k), upper 128 x TN tiles, K = n;
//   gram_rows  G = Z Z^T (n x n): K-major rows of H / L, K = m;
//   times      W = Z P^T (n x r, r <= 16): P (r x m) split into a 16-row
//              panel, one 128 x 16 tile per 128 rows of Z, K = m.
//
// Kernel (tc_split_kernel): one CTA of 128 threads per output tile.
//   warp 0 lane 0: TMA producer (cp.async.bulk.tensor, 128-byte swizzle, no
//                  multicast), an mbarrier ring of STAGES stages, each stage
//                  holding the H and L tiles of both operands;
//   warp 1 lane 0: MMA issuer: per 16-wide k step three
//                  tcgen05.mma.cta_group::1.kind::f16 (M = 128, N = TN) into
//                  one FP32 accumulator of TN TMEM columns; tcgen05.commit
//                  frees each stage;
//   warps 0-3:     epilogue: tcgen05.ld of the accumulator, stored
//                  column-major (C[col * ldc + row]) so that a warp's 32 rows
//                  form one 128-byte store.
// Every mbarrier wait is bounded.  A main-loop wait that expires sets the
// CTA's abort flag; the CTA then waits (bounded) for the MMAs and copies it
// has issued, frees its TMEM, and reports through *err, which the host turns
// into SYMPROP_ERR_TIMEOUT.  The epilogue's wait for the accumulator restarts
// its clock whenever the MMA issuer finishes a stage, so a long K axis is
// never mistaken for a stall.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include <atomic>
#include <cmath>
#include <mutex>

#include "common.cuh"
#include "gram_tc.cuh"

namespace spb {
namespace gram {

namespace {

constexpr int TM = 128;
constexpr uint64_t kWaitNs = 2000000000ull;  // bound of every wait (2 s)
// bound of the producer's and MMA issuer's waits; lowered only by the
// failure-injection hook symprop_debug_set_tc_wait_ns
std::atomic<uint64_t> g_mainloop_wait_ns{kWaitNs};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// bounded wait: false after `limit` ns, or as soon as another role aborts
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, volatile int *abort_flag,
                                          uint64_t limit) {
  const uint64_t t0 = global_ns();
  while (true) {
    if (mbar_try_wait(bar, parity)) return true;
    if (*abort_flag) return false;
    if (global_ns() - t0 > limit) return false;
  }
}

// wait for the accumulator: the clock restarts whenever *progress moves
__device__ __forceinline__ bool mbar_wait_progress(uint64_t *bar, volatile int *progress) {
  uint64_t t0 = global_ns();
  int seen = *progress;
  while (true) {
    if (mbar_try_wait(bar, 0)) return true;
    const int now = *progress;
    if (now != seen) {
      seen = now;
      t0 = global_ns();
    } else if (global_ns() - t0 > kWaitNs) {
      return false;
    }
  }
}

__device__ __forceinline__ void tma_load_2d(void *smem_dst, const CUtensorMap *map, uint64_t *bar,
                                            int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4}], [%2];" ::"r"(smem_u32(smem_dst)),
      "l"((uint64_t)map), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

// SM100 shared-memory matrix descriptor, 128-byte swizzle, version 1.
//   K-major: rows of 128 bytes (64 BF16 along k), 8-row groups 1024 B apart
//            (stride byte offset); the leading offset is unused.
//   MN-major: 128-byte rows along M/N, one row per k; 8-k groups 1024 B
//            apart (stride byte offset), 64-element M/N blocks `lbo` bytes
//            apart (leading byte offset).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)(1024 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
  return d;
}

// instruction descriptor of kind::f16: D = F32, A = B = BF16, M = 128
template <int TN, bool A_MN, bool B_MN>
constexpr uint32_t idesc() {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((A_MN ? 1u : 0u) << 15) | ((B_MN ? 1u : 0u) << 16) |
         ((uint32_t)(TN >> 3) << 17) | ((uint32_t)(TM >> 4) << 24);
}

template <uint32_t IDESC>
__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t acc) {
  uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(IDESC), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z));
}

__device__ __forceinline__ void umma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}

template <int W>
__device__ __forceinline__ void tmem_load(uint32_t taddr, uint32_t (&v)[W]);
template <>
__device__ __forceinline__ void tmem_load<32>(uint32_t taddr, uint32_t (&v)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,"
      "%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
        "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
        "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]),
        "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]),
        "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(taddr));
}
template <>
__device__ __forceinline__ void tmem_load<16>(uint32_t taddr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,"
      "%15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
        "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
        "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
}

struct TcArgs {
  int kblocks;                 // BK-wide blocks along K
  int rows_valid, cols_valid;  // output extent (rows of A, rows of B)
  float *C;                    // column-major output, C[col * ldc + row]
  size_t ldc;
  const int2 *tiles;           // (row tile, col tile) per tile; null: (CTA, 0)
  int ntiles;                  // tiles in the list
  int kb_per_split;            // K split: CTA u computes tile u % ntiles over the
  size_t split_stride;         // k blocks of split u / ntiles into C + split * split_stride
  int *err;                    // set to 1 when a wait expired
  uint64_t wait_ns;            // bound of the main-loop waits
};

// Shape of one operand tile in shared memory.
//   MN-major: BK rows of 128 bytes per 64-wide block, ROWS/64 blocks;
//   K-major:  ROWS rows of 128 bytes (BK = 64).
template <int ROWS, bool MN, int BK>
struct TileShape {
  static constexpr uint32_t box_bytes = MN ? (uint32_t)BK * 128u : (uint32_t)ROWS * 128u;
  static constexpr int boxes = MN ? ROWS / 64 : 1;
  static constexpr uint32_t bytes = box_bytes * boxes;
  static constexpr uint32_t lbo = MN ? box_bytes : 16u;
  static constexpr uint32_t kstep = MN ? 16u * 128u : 32u;  // bytes per 16-wide k step
  static_assert(MN ? (ROWS % 64 == 0) : (BK == 64), "tile shape");
};

template <int TN, bool A_MN, bool B_MN, int BK, int STAGES>
struct TcConfig {
  using TA = TileShape<TM, A_MN, BK>;
  using TB = TileShape<TN, B_MN, BK>;
  static constexpr uint32_t stage_bytes = 2 * TA::bytes + 2 * TB::bytes;
  static constexpr uint32_t tmem_cols = TN <= 32 ? 32u : (TN <= 64 ? 64u : (TN <= 128 ? 128u : 256u));
  static constexpr size_t smem = (size_t)STAGES * stage_bytes + 1024;
  static_assert(smem <= 227 * 1024, "shared memory");
  static_assert(TN % 16 == 0 && TN >= 16 && TN <= 256, "UMMA N");
};

template <int ROWS, bool MN, int BK>
__device__ __forceinline__ void load_tile(unsigned char *dst, const CUtensorMap *map, uint64_t *bar,
                                          int row0, int kb) {
  using T = TileShape<ROWS, MN, BK>;
  if (MN) {
#pragma unroll
    for (int b = 0; b < T::boxes; ++b) tma_load_2d(dst + b * T::box_bytes, map, bar, row0 + 64 * b, kb * BK);
  } else {
    tma_load_2d(dst, map, bar, kb * BK, row0);
  }
}

template <int TN, bool A_MN, bool B_MN, int BK, int STAGES>
__global__ void __launch_bounds__(128, 1)
    tc_split_kernel(const __grid_constant__ CUtensorMap mAh, const __grid_constant__ CUtensorMap mAl,
                    const __grid_constant__ CUtensorMap mBh, const __grid_constant__ CUtensorMap mBl,
                    const TcArgs a) {
  using Cfg = TcConfig<TN, A_MN, B_MN, BK, STAGES>;
  using TA = typename Cfg::TA;
  using TB = typename Cfg::TB;
  constexpr uint32_t IDESC = idesc<TN, A_MN, B_MN>();
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char *smem = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  __shared__ __align__(8) uint64_t full_bar[STAGES], empty_bar[STAGES], done_bar;
  __shared__ uint32_t tmem_base_holder;
  __shared__ volatile int abort_flag;
  __shared__ volatile int progress;
  __shared__ int issued[STAGES];

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int unit = (int)blockIdx.x;
  const int split = a.tiles ? unit / a.ntiles : 0;
  const int2 tile = a.tiles ? a.tiles[unit - split * a.ntiles] : make_int2(unit, 0);
  const int row0 = tile.x * TM, col0 = tile.y * TN;
  const int kb0 = split * a.kb_per_split;
  const int nkb = max(0, min(a.kblocks, kb0 + a.kb_per_split) - kb0);
  float *const C = a.C + (size_t)split * a.split_stride;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
      issued[s] = 0;
    }
    mbar_init(&done_bar, 1);
    abort_flag = 0;
    progress = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&tmem_base_holder)),
                 "r"(Cfg::tmem_cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = tmem_base_holder;

  auto stage_ptr = [&](int s) { return smem + (size_t)s * Cfg::stage_bytes; };

  if (warp == 0 && lane == 0) {
    // producer: H and L tiles of both operands per stage
    for (int it = 0; it < nkb; ++it) {
      const int s = it % STAGES;
      const uint32_t round = (uint32_t)(it / STAGES);
      if (it >= STAGES && !mbar_wait(&empty_bar[s], (round - 1) & 1, &abort_flag, a.wait_ns)) {
        abort_flag = 1;
        break;
      }
      unsigned char *st = stage_ptr(s);
      mbar_expect_tx(&full_bar[s], Cfg::stage_bytes);
      const int kb = kb0 + it;
      load_tile<TM, A_MN, BK>(st, &mAh, &full_bar[s], row0, kb);
      load_tile<TM, A_MN, BK>(st + TA::bytes, &mAl, &full_bar[s], row0, kb);
      load_tile<TN, B_MN, BK>(st + 2 * TA::bytes, &mBh, &full_bar[s], col0, kb);
      load_tile<TN, B_MN, BK>(st + 2 * TA::bytes + TB::bytes, &mBl, &full_bar[s], col0, kb);
      issued[s] = it + 1;
    }
  } else if (warp == 1 && lane == 0) {
    // MMA issuer: Ah Bh^T + Ah Bl^T + Al Bh^T per 16-wide k step
    bool ok = true;
    for (int it = 0; it < nkb; ++it) {
      const int s = it % STAGES;
      const uint32_t round = (uint32_t)(it / STAGES);
      if (!mbar_wait(&full_bar[s], round & 1, &abort_flag, a.wait_ns)) {
        abort_flag = 1;
        ok = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;");
      const uint32_t base = smem_u32(stage_ptr(s));
      const uint32_t ah = base, al = base + TA::bytes, bh = base + 2 * TA::bytes,
                     bl = base + 2 * TA::bytes + TB::bytes;
#pragma unroll
      for (int k = 0; k < BK / 16; ++k) {
        const uint64_t dah = smem_desc(ah + k * TA::kstep, TA::lbo);
        const uint64_t dal = smem_desc(al + k * TA::kstep, TA::lbo);
        const uint64_t dbh = smem_desc(bh + k * TB::kstep, TB::lbo);
        const uint64_t dbl = smem_desc(bl + k * TB::kstep, TB::lbo);
        umma_bf16<IDESC>(tmem, dah, dbh, (it > 0 || k > 0) ? 1u : 0u);
        umma_bf16<IDESC>(tmem, dah, dbl, 1u);
        umma_bf16<IDESC>(tmem, dal, dbh, 1u);
      }
      umma_commit(&empty_bar[s]);
      progress = it + 1;
    }
    // completion of every MMA issued, also after an abort, so that TMEM is
    // never freed under an MMA in flight
    umma_commit(&done_bar);
    if (!ok) abort_flag = 1;
  }
  __syncwarp();
  const bool done = mbar_wait_progress(&done_bar, &progress);
  asm volatile("tcgen05.fence::after_thread_sync;");
  const int go = __all_sync(0xffffffffu, done ? 1 : 0) && !__shfl_sync(0xffffffffu, (int)abort_flag, 0) &&
                 nkb > 0;
  if (go) {
    const int r = row0 + warp * 32 + lane;
    constexpr int W = TN < 32 ? TN : 32;
#pragma unroll 1
    for (int c = 0; c < TN; c += W) {
      uint32_t v[W];
      tmem_load<W>(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (r < a.rows_valid) {
#pragma unroll
        for (int j = 0; j < W; ++j) {
          const int col = col0 + c + j;
          if (col < a.cols_valid) C[(size_t)col * a.ldc + r] = __uint_as_float(v[j]);
        }
      }
    }
  } else if (threadIdx.x == 0) {
    atomicExch(a.err, 1);
  }
  // teardown: the copies issued into this CTA's shared memory land before it
  // exits (they were issued whether or not an MMA consumed them)
  if (threadIdx.x == 0 && (abort_flag || !done)) {
    for (int s = 0; s < STAGES; ++s) {
      if (issued[s] > 0) {
        volatile int never = 0;
        mbar_wait(&full_bar[s], (uint32_t)((issued[s] - 1) / STAGES) & 1, (volatile int *)&never, kWaitNs);
      }
    }
    if (!done) {
      volatile int never = 0;
      mbar_wait(&done_bar, 0, (volatile int *)&never, kWaitNs);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(Cfg::tmem_cols));
  }
}

// Z = X diag(colscale) split into H = bf16(Z), L = bf16(Z - H), row-major
// rows x ld with zero padding past `cols`.  Each thread writes 8 columns.
__global__ void split_rows_kernel(const float *__restrict__ X, int rows, int cols,
                                  const float *__restrict__ colscale, __nv_bfloat16 *__restrict__ H,
                                  __nv_bfloat16 *__restrict__ L, int ld) {
  const int groups = ld / 8;
  const size_t id = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= (size_t)rows * groups) return;
  const int r = (int)(id / groups), c0 = (int)(id % groups) * 8;
  alignas(16) __nv_bfloat16 h[8], l[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const int c = c0 + j;
    const float z = c < cols ? X[(size_t)r * cols + c] * (colscale ? colscale[c] : 1.f) : 0.f;
    h[j] = __float2bfloat16_rn(z);
    l[j] = __float2bfloat16_rn(z - __bfloat162float(h[j]));
  }
  *(uint4 *)(H + (size_t)r * ld + c0) = *(const uint4 *)h;
  *(uint4 *)(L + (size_t)r * ld + c0) = *(const uint4 *)l;
}

// Panel of a product W = Z P^T: Bh / Bl (rows_pad x ld) = split of
// P[q * sq + k * sk] * colscale[k] for q < r, k < cols, zero elsewhere.
__global__ void split_panel_kernel(const double *__restrict__ P, int r, int cols, size_t sq, size_t sk,
                                   const double *__restrict__ colscale, __nv_bfloat16 *__restrict__ Bh,
                                   __nv_bfloat16 *__restrict__ Bl, int rows_pad, int ld) {
  const size_t id = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= (size_t)rows_pad * ld) return;
  const int q = (int)(id / ld), k = (int)(id % ld);
  float z = 0.f;
  if (q < r && k < cols) z = (float)(P[q * sq + k * sk] * (colscale ? colscale[k] : 1.0));
  const __nv_bfloat16 h = __float2bfloat16_rn(z);
  Bh[id] = h;
  Bl[id] = __float2bfloat16_rn(z - __bfloat162float(h));
}

// S (n x n FP64, full symmetric) from the column-major upper tiles of G
// summed over the K splits: Gc[s][col * n + row] holds split s of G[row][col]
// for row <= col; the splits are added in FP64, in split order.
__global__ void symmetrize_kernel(const float *__restrict__ Gc, int n, int splits, double *__restrict__ S) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t nn = (size_t)n * n;
  if (idx >= nn) return;
  const int i = (int)(idx / n), j = (int)(idx % n);
  const size_t at = i <= j ? (size_t)j * n + i : (size_t)i * n + j;
  double v = 0.0;
  for (int sp = 0; sp < splits; ++sp) v += (double)Gc[sp * nn + at];
  S[idx] = v;
}

// W (rows x r FP64, row stride ldw) from the column-major product Wc (16 columns of `rows`)
__global__ void gather_panel_kernel(const float *__restrict__ Wc, int rows, int r, double *__restrict__ W,
                                    size_t ldw) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (size_t)rows * r) return;
  const int i = (int)(idx / r), q = (int)(idx % r);
  W[(size_t)i * ldw + q] = (double)Wc[(size_t)q * rows + i];
}

// Upper-triangular tile list of a Gram of dimension dim in 128 x tn tiles:
// row tile i keeps the column tiles j >= floor(128 i / tn) (those that reach
// the upper triangle), in row-major order.  One thread per tile.
__host__ __device__ inline int first_upper_col(int i, int tn) { return (i * TM) / tn; }

__global__ void upper_tiles_kernel(int2 *tiles, int nt_r, int nt_c, int tn, int count) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  int base = 0;
  for (int i = 0; i < nt_r; ++i) {
    const int j0 = first_upper_col(i, tn), per = nt_c - j0;
    if (t < base + per) {
      tiles[t] = make_int2(i, j0 + (t - base));
      return;
    }
    base += per;
  }
}

PFN_cuTensorMapEncodeTiled_v12000 get_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  });
  if (!fn) fail(SYMPROP_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable");
  return fn;
}

// 2-D map over a row-major BF16 matrix (rows x ld elements), box {64, box_rows}
CUtensorMap make_map(const __nv_bfloat16 *base, int rows, int ld, int box_rows) {
  if (((uintptr_t)base & 15) || (ld % 8)) fail(SYMPROP_ERR_INVALID, "tensor map: misaligned operand");
  CUtensorMap map;
  cuuint64_t dims[2] = {(cuuint64_t)ld, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
  cuuint32_t box[2] = {64u, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = get_encoder()(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, (void *)base, dims, strides,
                             box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) fail(SYMPROP_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return map;
}

template <int TN, bool A_MN, bool B_MN, int BK, int STAGES>
void launch(cudaStream_t st, const CUtensorMap &ah, const CUtensorMap &al, const CUtensorMap &bh,
            const CUtensorMap &bl, const TcArgs &a, unsigned ctas) {
  using Cfg = TcConfig<TN, A_MN, B_MN, BK, STAGES>;
  auto k = tc_split_kernel<TN, A_MN, B_MN, BK, STAGES>;
  SPB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Cfg::smem));
  if (ctas) k<<<ctas, 128, Cfg::smem, st>>>(ah, al, bh, bl, a);
  SPB_LAUNCH_CHECK();
}

// Gram tiles: 128 x 256 for the m x m product (MN-major operands, BK = 32,
// 48 KB per stage), 128 x 128 for the n x n product (K-major, BK = 64, one
// map for both operands, 64 KB per stage)
constexpr int kColsTN = 256, kColsBK = 32, kColsStages = 4;
constexpr int kRowsTN = 128, kRowsStages = 3;
constexpr int kPanelStages = 5;  // 36 KB per stage
// K splits of a Gram: at least this many k blocks per split
constexpr int kMinKbPerSplit = 64;
constexpr int kMaxSplits = 8;

size_t up256(size_t x) { return (x + 255) / 256 * 256; }

}  // namespace

uint64_t mainloop_wait_ns() { return g_mainloop_wait_ns.load(); }
void set_mainloop_wait_ns(uint64_t ns) { g_mainloop_wait_ns.store(ns ? ns : kWaitNs); }

int split_ld(int cols) { return (cols + 63) / 64 * 64; }

size_t split_bytes(int rows, int cols) { return 2 * up256((size_t)rows * split_ld(cols) * 2); }

Split split_view(void *ws, int rows, int cols) {
  Split z;
  z.rows = rows;
  z.cols = cols;
  z.ld = split_ld(cols);
  z.h = (__nv_bfloat16 *)ws;
  z.l = (__nv_bfloat16 *)((unsigned char *)ws + up256((size_t)rows * z.ld * 2));
  return z;
}

void split(cudaStream_t st, const float *X, const float *colscale, const Split &z) {
  const size_t work = (size_t)z.rows * (z.ld / 8);
  if (!work) return;
  split_rows_kernel<<<(unsigned)((work + 255) / 256), 256, 0, st>>>(X, z.rows, z.cols, colscale, z.h, z.l,
                                                                   z.ld);
  SPB_LAUNCH_CHECK();
}

namespace {

int sm_count() {
  int dev = 0, sms = 0;
  SPB_CUDA(cudaGetDevice(&dev));
  SPB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  return sms > 0 ? sms : 1;
}

// Work of one Gram: its upper tiles and the K splits.  The split count
// makes the last wave of CTAs as full as it can (up to kMaxSplits, each
// split at least kMinKbPerSplit k blocks; ties go to more splits, which
// also shortens each FP32 accumulation chain).
struct GramPlan {
  int dim, tn, nt, ntc, ntiles, kblocks, splits, kb_per_split;
};

GramPlan plan_gram(const Split &z, bool cols_mode) {
  GramPlan g;
  g.dim = cols_mode ? z.cols : z.rows;
  g.tn = cols_mode ? kColsTN : kRowsTN;
  g.nt = (g.dim + TM - 1) / TM;
  g.ntc = (g.dim + g.tn - 1) / g.tn;
  g.ntiles = 0;
  for (int i = 0; i < g.nt; ++i) g.ntiles += g.ntc - first_upper_col(i, g.tn);
  g.kblocks = cols_mode ? (z.rows + kColsBK - 1) / kColsBK : z.ld / 64;
  const int sms = sm_count();
  auto fill = [&](int sp) {
    const double units = (double)g.ntiles * sp;
    return units / (std::ceil(units / sms) * sms);
  };
  int best = 1;
  double best_fill = fill(1);
  for (int sp = 2; sp <= kMaxSplits && g.kblocks / sp >= kMinKbPerSplit; ++sp)
    if (fill(sp) >= best_fill - 0.005) {
      best = sp;
      best_fill = std::max(best_fill, fill(sp));
    }
  g.kb_per_split = std::max(1, (g.kblocks + best - 1) / best);
  g.splits = std::max(1, (g.kblocks + g.kb_per_split - 1) / g.kb_per_split);
  return g;
}

size_t plan_scratch_bytes(const GramPlan &g) {
  return up256((size_t)g.splits * g.dim * g.dim * 4) + up256((size_t)g.ntiles * sizeof(int2)) + 256;
}

Split shape_only(int rows, int cols) {
  Split z;
  z.rows = rows;
  z.cols = cols;
  z.ld = split_ld(cols);
  return z;
}

// G (dim x dim) from its upper tiles; `cols_mode` picks G = Z^T Z (dim = m,
// MN-major operands) or G = Z Z^T (dim = n, K-major operands).
void gram(cudaStream_t st, const Split &z, bool cols_mode, double *S, void *scratch, int *d_err) {
  const GramPlan g = plan_gram(z, cols_mode);
  if (g.dim <= 0 || g.ntiles <= 0) return;
  unsigned char *w = (unsigned char *)scratch;
  float *Gc = (float *)w;
  int2 *tiles = (int2 *)(w + up256((size_t)g.splits * g.dim * g.dim * 4));
  // the tile list is written on the device (no host staging, fixed order)
  upper_tiles_kernel<<<(unsigned)((g.ntiles + 127) / 128), 128, 0, st>>>(tiles, g.nt, g.ntc, g.tn, g.ntiles);
  SPB_LAUNCH_CHECK();
  TcArgs a;
  a.rows_valid = a.cols_valid = g.dim;
  a.C = Gc;
  a.ldc = (size_t)g.dim;
  a.tiles = tiles;
  a.ntiles = g.ntiles;
  a.kblocks = g.kblocks;
  a.kb_per_split = g.kb_per_split;
  a.split_stride = (size_t)g.dim * g.dim;
  a.err = d_err;
  a.wait_ns = mainloop_wait_ns();
  const unsigned ctas = (unsigned)(g.ntiles * g.splits);
  if (cols_mode) {
    // operands: 64-wide column strips of H / L, kColsBK rows of k per box
    CUtensorMap h = make_map(z.h, z.rows, z.ld, kColsBK), l = make_map(z.l, z.rows, z.ld, kColsBK);
    launch<kColsTN, true, true, kColsBK, kColsStages>(st, h, l, h, l, a, ctas);
  } else {
    static_assert(kRowsTN == TM, "one map serves both operands of the row Gram");
    CUtensorMap h = make_map(z.h, z.rows, z.ld, TM), l = make_map(z.l, z.rows, z.ld, TM);
    launch<kRowsTN, false, false, 64, kRowsStages>(st, h, l, h, l, a, ctas);
  }
  symmetrize_kernel<<<(unsigned)(((size_t)g.dim * g.dim + 255) / 256), 256, 0, st>>>(Gc, g.dim, g.splits, S);
  SPB_LAUNCH_CHECK();
}

}  // namespace

size_t gram_cols_scratch_bytes(int rows, int cols) {
  return plan_scratch_bytes(plan_gram(shape_only(rows, cols), true));
}

size_t gram_rows_scratch_bytes(int rows, int cols) {
  return plan_scratch_bytes(plan_gram(shape_only(rows, cols), false));
}

void gram_cols(cudaStream_t st, const Split &z, double *S, void *scratch, int *d_err) {
  gram(st, z, true, S, scratch, d_err);
}

void gram_rows(cudaStream_t st, const Split &z, double *S, void *scratch, int *d_err) {
  gram(st, z, false, S, scratch, d_err);
}

size_t times_scratch_bytes(int rows, int cols) {
  return up256((size_t)kPanelRows * rows * 4) + 2 * up256((size_t)kPanelRows * split_ld(cols) * 2);
}

void times(cudaStream_t st, const Split &z, const double *P, int r, size_t sq, size_t sk,
           const double *colscale, double *W, size_t ldw, void *scratch, int *d_err) {
  if (r < 1 || r > kPanelRows) fail(SYMPROP_ERR_SIZE, "tensor-core panel product: r = %d (1..%d)", r, kPanelRows);
  if (z.rows <= 0) return;
  unsigned char *w = (unsigned char *)scratch;
  float *Wc = (float *)w;
  __nv_bfloat16 *bh = (__nv_bfloat16 *)(w + up256((size_t)kPanelRows * z.rows * 4));
  __nv_bfloat16 *bl = (__nv_bfloat16 *)((unsigned char *)bh + up256((size_t)kPanelRows * z.ld * 2));
  const size_t pw = (size_t)kPanelRows * z.ld;
  split_panel_kernel<<<(unsigned)((pw + 255) / 256), 256, 0, st>>>(P, r, z.cols, sq, sk, colscale, bh, bl,
                                                                  kPanelRows, z.ld);
  SPB_LAUNCH_CHECK();
  CUtensorMap ha = make_map(z.h, z.rows, z.ld, TM), la = make_map(z.l, z.rows, z.ld, TM);
  CUtensorMap hb = make_map(bh, kPanelRows, z.ld, kPanelRows), lb = make_map(bl, kPanelRows, z.ld, kPanelRows);
  TcArgs a;
  a.kblocks = z.ld / 64;
  a.rows_valid = z.rows;
  a.cols_valid = kPanelRows;
  a.C = Wc;
  a.ldc = (size_t)z.rows;
  a.tiles = nullptr;
  a.ntiles = (z.rows + TM - 1) / TM;
  a.kb_per_split = a.kblocks;
  a.split_stride = 0;
  a.err = d_err;
  a.wait_ns = mainloop_wait_ns();
  launch<kPanelRows, false, false, 64, kPanelStages>(st, ha, la, hb, lb, a, (unsigned)((z.rows + TM - 1) / TM));
  gather_panel_kernel<<<(unsigned)(((size_t)z.rows * r + 255) / 256), 256, 0, st>>>(Wc, z.rows, r, W, ldw);
  SPB_LAUNCH_CHECK();
}

size_t workspace_bytes(int n, int m) { return split_bytes(n, m) + gram_cols_scratch_bytes(n, m); }

void gram_split_bf16(cudaStream_t st, const float *Y, int n, int m, const float *sd, double *S, void *ws,
                     int *d_err) {
  if (n <= 0 || m <= 0) return;
  Split z = split_view(ws, n, m);
  split(st, Y, sd, z);
  gram_cols(st, z, S, (unsigned char *)ws + split_bytes(n, m), d_err);
}

// ---------------------------------------------------------------------------
// Allocation-free Gram.  Some callers cannot allocate device memory when
// they call this library: services that reserve all device memory for their
// own pool allocator at start-up (a later cudaMalloc fails or fragments the
// pool), and code that must not pay cudaMalloc/cudaFree's implicit device
// synchronisation.  For them the workspace of the tensor-core Gram lives in
// one file-scope device array of kNoAllocBytes (32 MiB), which every GPU
// that loads this library holds until the process exits.  The kernels and
// their launch parameters are the ones of gram_split_bf16, so the two entry
// points give the same matrix bit for bit.
namespace {

constexpr size_t kNoAllocBytes = 32ull << 20;
__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

std::mutex g_noalloc_mu;
void *g_noalloc_ptr[64] = {};

// Device address of the scratch array on `device`, which must be current.
// It is looked up once per device, at the first call there, and kept: a
// device reset (cudaDeviceReset, or a reset primary context) invalidates it,
// so this entry point must not be used across one.
void *noalloc_scratch(int device) {
  if (device < 0 || device >= 64) fail(SYMPROP_ERR_INVALID, "device id %d out of range", device);
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[device]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      fail(SYMPROP_ERR_CUDA, "cudaGetSymbolAddress(g_noalloc_scratch) failed: %s", cudaGetErrorString(e));
    }
    g_noalloc_ptr[device] = p;
  }
  return g_noalloc_ptr[device];
}

}  // namespace

size_t noalloc_capacity() { return kNoAllocBytes; }

void gram_split_bf16_noalloc(cudaStream_t st, const float *Y, int n, int m, const float *sd, double *S) {
  if (n <= 0 || m <= 0) fail(SYMPROP_ERR_INVALID, "n and m must be positive");
  // layout: split operands | Gram scratch | error flag
  const size_t need = workspace_bytes(n, m) + 256;
  if (need > kNoAllocBytes)
    fail(SYMPROP_ERR_SIZE,
         "allocation-free Gram: n=%d, m=%d needs %zu bytes of scratch, the fixed array holds %zu", n, m,
         need, kNoAllocBytes);
  int dev = 0;
  SPB_CUDA(cudaGetDevice(&dev));
  unsigned char *w = (unsigned char *)noalloc_scratch(dev);
  int *err = (int *)(w + workspace_bytes(n, m));
  SPB_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));  // the array keeps the previous call's contents
  gram_split_bf16(st, Y, n, m, sd, S, w, err);
  int h = 0;
  SPB_CUDA(cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, st));
  SPB_CUDA(cudaStreamSynchronize(st));
  if (h) fail(SYMPROP_ERR_TIMEOUT, "tensor-core Gram: a bounded wait expired");
}

}  // namespace gram
}  // namespace spb

// See include/symprop.h: allocation-free tensor-core Gram.
extern "C" int symprop_gram_device_noalloc(const float *dY, uint64_t n, uint32_t m, const float *dscale,
                                           double *dG, void *stream) {
  return spb::guard([&] {
    if (!dY || !dscale || !dG) spb::fail(SYMPROP_ERR_INVALID, "null argument");
    if (n == 0 || m == 0 || n >= (1ull << 31)) spb::fail(SYMPROP_ERR_INVALID, "bad sizes");
    spb::gram::gram_split_bf16_noalloc((cudaStream_t)stream, dY, (int)n, (int)m, dscale, dG);
  });
}

// See include/symprop.h: failure-injection hook of the tensor-core kernels.
extern "C" int symprop_debug_set_tc_wait_ns(uint64_t ns) {
  spb::gram::set_mainloop_wait_ns(ns);
  return SYMPROP_OK;
}
