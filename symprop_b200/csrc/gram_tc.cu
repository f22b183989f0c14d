// Packed Gram matrix G = D^1/2 Y^T Y D^1/2 on the 5th-generation tensor
// cores (tcgen05), split-BF16 operands with FP32 accumulation in TMEM.
//
// This is the mixed-precision form of HOOI's dense step: the reference takes
// the left singular vectors of the unpacked Y with dgesvd
// (src/sparse/spsymtensor.cpp:225, src/dense/matrixops.cpp:18-43); their span
// is the top-r eigenspace of the m x m packed Gram (see tucker.cu).
//
// Y' = Y D^1/2 (FP32) is split as Y' ~ H + L with H = bf16(Y'),
// L = bf16(Y' - H); G ~ H^T H + H^T L + L^T H (the L^T L term, 2^-16
// relative, is dropped).  The three products are one GEMM over a K axis of
// 3n: A = [H | H | L], B = [H | L | H] (K-major tiles of H^T, L^T).
//
// Kernel: one CTA per 128 x 128 upper-triangular tile of G, 128 threads.
//   warp 0 lane 0: TMA producer (cp.async.bulk.tensor, 128B swizzle,
//                  6-stage mbarrier ring; each CTA loads its own tiles)
//   warp 1 lane 0: MMA issuer (tcgen05.mma.cta_group::1.kind::f16, M=N=128,
//                  K=16 per instruction, accumulator in 128 TMEM columns;
//                  tcgen05.commit releases each smem stage)
//   warps 0-3:     epilogue (tcgen05.ld 32x32b.x32 -> FP32 stores)
// Every mbarrier wait is bounded; on expiry the CTA records an error, waits
// (bounded) for its in-flight copies, frees its TMEM and returns.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include <mutex>

#include "common.cuh"
#include "gram_tc.cuh"

namespace spb {
namespace gram {

namespace {

constexpr int TM = 128, TN = 128, BK = 64, STAGES = 6;
constexpr uint32_t STAGE_BYTES = (TM + TN) * BK * 2;  // 32 KB
constexpr uint32_t TMEM_COLS = 128;
constexpr uint64_t kWaitNs = 2000000000ull;  // bound of every mbarrier wait (2 s)

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

// bounded wait: false after kWaitNs or when another role has aborted
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, volatile int *abort_flag) {
  const uint64_t t0 = global_ns();
  while (true) {
    if (mbar_try_wait(bar, parity)) return true;
    if (*abort_flag) return false;
    if (global_ns() - t0 > kWaitNs) return false;
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

// SM100 shared-memory matrix descriptor: K-major, 128B swizzle, 8-row
// groups 1024 B apart (SBO), version 1.
__device__ __forceinline__ uint64_t smem_desc(const void *p) {
  uint64_t addr = smem_u32(p);
  uint64_t d = 0;
  d |= (addr >> 4) & 0x3FFFull;          // start address
  d |= (uint64_t)1 << 16;                 // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(1024 >> 4) << 32;       // stride byte offset
  d |= (uint64_t)1 << 46;                 // version
  d |= (uint64_t)2 << 61;                 // SWIZZLE_128B
  return d;
}

// instruction descriptor: D=F32, A=B=BF16, K-major both, N=128, M=128
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TN >> 3) << 17) |
                            ((uint32_t)(TM >> 4) << 24);

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t acc) {
  uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(kIdesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z));
}

__device__ __forceinline__ void umma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}

__global__ void __launch_bounds__(128, 1)
    gram_tile_kernel(const __grid_constant__ CUtensorMap mapH, const __grid_constant__ CUtensorMap mapL,
                     const int2 *__restrict__ tiles, int m, int kblocks, float *__restrict__ G,
                     int *__restrict__ err) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // 1024-byte aligned stage buffers (the swizzle pattern assumes it)
  unsigned char *smem = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  unsigned char *sA = smem;
  unsigned char *sB = smem + STAGES * TM * BK * 2;
  __shared__ __align__(8) uint64_t full_bar[STAGES], empty_bar[STAGES], done_bar;
  __shared__ uint32_t tmem_base_holder;
  __shared__ volatile int abort_flag;
  __shared__ int issued[STAGES];

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int2 tile = tiles[blockIdx.x];
  const int row0 = tile.x * TM, col0 = tile.y * TN;
  const int total = 3 * kblocks;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
      issued[s] = 0;
    }
    mbar_init(&done_bar, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&tmem_base_holder)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = tmem_base_holder;

  if (warp == 0 && lane == 0) {
    // producer
    for (int it = 0; it < total; ++it) {
      const int s = it % STAGES;
      const uint32_t round = (uint32_t)(it / STAGES);
      if (it >= STAGES) {
        if (!mbar_wait(&empty_bar[s], (round - 1) & 1, &abort_flag)) {
          abort_flag = 1;
          break;
        }
      }
      const int seg = it / kblocks, kb = it - seg * kblocks;
      const CUtensorMap *ma = (seg == 2) ? &mapL : &mapH;
      const CUtensorMap *mb = (seg == 1) ? &mapL : &mapH;
      mbar_expect_tx(&full_bar[s], STAGE_BYTES);
      tma_load_2d(sA + s * TM * BK * 2, ma, &full_bar[s], kb * BK, row0);
      tma_load_2d(sB + s * TN * BK * 2, mb, &full_bar[s], kb * BK, col0);
      issued[s] = it + 1;
    }
  } else if (warp == 1 && lane == 0) {
    // MMA issuer
    bool ok = true;
    for (int it = 0; it < total; ++it) {
      const int s = it % STAGES;
      const uint32_t round = (uint32_t)(it / STAGES);
      if (!mbar_wait(&full_bar[s], round & 1, &abort_flag)) {
        abort_flag = 1;
        ok = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;");
      const unsigned char *a = sA + s * TM * BK * 2, *b = sB + s * TN * BK * 2;
      const uint64_t da = smem_desc(a), db = smem_desc(b);
#pragma unroll
      for (int k = 0; k < BK / 16; ++k) {
        // advance 16 BF16 (32 bytes) along K inside the swizzle atom
        umma_bf16(tmem, da + (uint64_t)(k * 2), db + (uint64_t)(k * 2), (it > 0 || k > 0) ? 1u : 0u);
      }
      umma_commit(&empty_bar[s]);
    }
    // always signal completion of every MMA issued, so TMEM is never freed
    // under an in-flight MMA
    umma_commit(&done_bar);
    if (!ok) abort_flag = 1;
  }
  __syncwarp();
  // epilogue: wait for the accumulator (the wait itself ignores aborts so
  // that issued MMAs always drain first)
  volatile int no_abort = 0;
  bool ok = mbar_wait(&done_bar, 0, &no_abort);
  asm volatile("tcgen05.fence::after_thread_sync;");
  const int go = __all_sync(0xffffffffu, ok ? 1 : 0) && !__shfl_sync(0xffffffffu, (int)abort_flag, 0);
  if (go) {
    const int r = row0 + warp * 32 + lane;
#pragma unroll 1
    for (int c = 0; c < TN; c += 32) {
      uint32_t v[32];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,"
          "%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
            "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
            "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]),
            "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]),
            "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (r < m) {
#pragma unroll
        for (int j = 0; j < 32; ++j) {
          const int col = col0 + c + j;
          if (col < m) G[(size_t)r * m + col] = __uint_as_float(v[j]);
        }
      }
    }
  } else if (threadIdx.x == 0) {
    atomicExch(err, 1);
  }
  // teardown: let in-flight copies land before the CTA's smem goes away
  if (threadIdx.x == 0 && abort_flag) {
    for (int s = 0; s < STAGES; ++s) {
      if (issued[s] > 0) {
        const uint32_t round = (uint32_t)((issued[s] - 1) / STAGES);
        volatile int never = 0;
        mbar_wait(&full_bar[s], round & 1, (volatile int *)&never);
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
  }
}

// Y' = Y * sd (column scale) split into H, L (BF16), written K-major
// (transposed: out[col][row]) with leading dimension ldk.
__global__ void split_transpose_kernel(const float *__restrict__ Y, int n, int m,
                                       const float *__restrict__ sd, __nv_bfloat16 *H,
                                       __nv_bfloat16 *L, int ldk) {
  __shared__ float tile[32][33];
  const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    int r = r0 + i, c = c0 + threadIdx.x;
    tile[i][threadIdx.x] = (r < n && c < m) ? Y[(size_t)r * m + c] * sd[c] : 0.f;
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    int c = c0 + i, r = r0 + threadIdx.x;
    if (c < m && r < ldk) {
      float v = (r < n) ? tile[threadIdx.x][i] : 0.f;
      __nv_bfloat16 h = __float2bfloat16_rn(v);
      __nv_bfloat16 l = __float2bfloat16_rn(v - __bfloat162float(h));
      H[(size_t)c * ldk + r] = h;
      L[(size_t)c * ldk + r] = l;
    }
  }
}

// full symmetric FP64 matrix from the upper tiles
__global__ void symmetrize_kernel(const float *G, int m, double *S) {
  size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (size_t)m * m) return;
  int i = (int)(idx / m), j = (int)(idx % m);
  bool upper = i <= j;  // upper tiles are complete; i <= j also fixes the diagonal tiles
  S[idx] = (double)(upper ? G[idx] : G[(size_t)j * m + i]);
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

CUtensorMap make_map(const __nv_bfloat16 *base, int rows, int ldk, int kvalid) {
  CUtensorMap map;
  cuuint64_t dims[2] = {(cuuint64_t)kvalid, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)ldk * 2};
  cuuint32_t box[2] = {(cuuint32_t)BK, (cuuint32_t)TM};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = get_encoder()(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, (void *)base, dims, strides,
                             box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) fail(SYMPROP_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return map;
}

}  // namespace

size_t workspace_bytes(int n, int m) {
  const size_t ldk = ((size_t)n + 63) / 64 * 64;
  const int tiles = (m + TM - 1) / TM;
  return 2 * (size_t)m * ldk * 2 + (size_t)m * m * 4 + (size_t)tiles * (tiles + 1) / 2 * sizeof(int2) +
         4096;
}

void gram_split_bf16(cudaStream_t st, const float *Y, int n, int m, const float *sd, double *S,
                     void *ws, int *d_err) {
  if (n <= 0 || m <= 0) return;
  const int ldk = (n + 63) / 64 * 64;
  unsigned char *w = (unsigned char *)ws;
  __nv_bfloat16 *H = (__nv_bfloat16 *)w;
  __nv_bfloat16 *L = H + (size_t)m * ldk;
  float *G = (float *)(L + (size_t)m * ldk);
  int2 *tiles = (int2 *)(((uintptr_t)(G + (size_t)m * m) + 15) & ~(uintptr_t)15);
  const int nt = (m + TM - 1) / TM;
  std::vector<int2> ht;
  for (int i = 0; i < nt; ++i)
    for (int j = i; j < nt; ++j) ht.push_back(make_int2(i, j));
  SPB_CUDA(cudaMemcpyAsync(tiles, ht.data(), ht.size() * sizeof(int2), cudaMemcpyHostToDevice, st));
  dim3 tb(32, 8), tg((m + 31) / 32, (ldk + 31) / 32);
  split_transpose_kernel<<<tg, tb, 0, st>>>(Y, n, m, sd, H, L, ldk);
  SPB_LAUNCH_CHECK();
  CUtensorMap mH = make_map(H, m, ldk, ldk), mL = make_map(L, m, ldk, ldk);
  const int kblocks = ldk / BK;
  const size_t smem = (size_t)STAGES * STAGE_BYTES + 1024;
  SPB_CUDA(cudaFuncSetAttribute(gram_tile_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  gram_tile_kernel<<<(unsigned)ht.size(), 128, smem, st>>>(mH, mL, tiles, m, kblocks, G, d_err);
  SPB_LAUNCH_CHECK();
  symmetrize_kernel<<<(unsigned)(((size_t)m * m + 255) / 256), 256, 0, st>>>(G, m, S);
  SPB_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------------
// Allocation-free variant.  Some callers cannot allocate device memory when
// they call this library: services that reserve all device memory for their
// own pool allocator at start-up (a later cudaMalloc fails or fragments the
// pool), and code that must not pay cudaMalloc/cudaFree's implicit device
// synchronisation.  For them the workspace of the tensor-core Gram lives in
// one file-scope device array of kNoAllocBytes (32 MiB), which every GPU
// that loads this library holds until the process exits.
namespace {

constexpr size_t kNoAllocBytes = 32ull << 20;
__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// upper-triangular tile list written on the device (no host buffer)
__global__ void fill_tiles_kernel(int2 *tiles, int nt) {
  int id = blockIdx.x * blockDim.x + threadIdx.x;
  int k = 0;
  for (int i = 0; i < nt; ++i)
    for (int j = i; j < nt; ++j, ++k)
      if (k == id) tiles[id] = make_int2(i, j);
}

std::mutex g_noalloc_mu;
void *g_noalloc_ptr[64] = {};

// device address of the scratch array on the current device (looked up once
// per device, with that device current)
void *noalloc_scratch(int device) {
  if (device < 0 || device >= 64) fail(SYMPROP_ERR_INVALID, "device id %d out of range", device);
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[device]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      fail(SYMPROP_ERR_CUDA, "cudaGetSymbolAddress(g_noalloc_scratch) failed: %s", cudaGetErrorString(e));
    g_noalloc_ptr[device] = p;
  }
  return g_noalloc_ptr[device];
}

}  // namespace

size_t noalloc_capacity() { return kNoAllocBytes; }

void gram_split_bf16_noalloc(cudaStream_t st, const float *Y, int n, int m, const float *sd, double *S) {
  if (n <= 0 || m <= 0) fail(SYMPROP_ERR_INVALID, "n and m must be positive");
  const size_t ldk = ((size_t)n + 63) / 64 * 64;
  const int nt = (m + TM - 1) / TM;
  const size_t ntiles = (size_t)nt * (nt + 1) / 2;
  // layout: H | L | G (FP32) | tiles | error flag, each 256-byte aligned
  auto up = [](size_t x) { return (x + 255) / 256 * 256; };
  const size_t oH = 0, oL = up(oH + (size_t)m * ldk * 2), oG = up(oL + (size_t)m * ldk * 2),
               oT = up(oG + (size_t)m * m * 4), oE = up(oT + ntiles * sizeof(int2)), need = oE + 256;
  if (need > kNoAllocBytes)
    fail(SYMPROP_ERR_SIZE,
         "allocation-free Gram: n=%d, m=%d needs %zu bytes of scratch, the fixed array holds %zu", n, m,
         need, kNoAllocBytes);
  int dev = 0;
  SPB_CUDA(cudaGetDevice(&dev));
  unsigned char *w = (unsigned char *)noalloc_scratch(dev);
  __nv_bfloat16 *H = (__nv_bfloat16 *)(w + oH), *L = (__nv_bfloat16 *)(w + oL);
  float *G = (float *)(w + oG);
  int2 *tiles = (int2 *)(w + oT);
  int *err = (int *)(w + oE);
  SPB_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));  // the array keeps the previous call's contents
  fill_tiles_kernel<<<(unsigned)((ntiles + 127) / 128), 128, 0, st>>>(tiles, nt);
  SPB_LAUNCH_CHECK();
  dim3 tb(32, 8), tg((m + 31) / 32, (unsigned)((ldk + 31) / 32));
  split_transpose_kernel<<<tg, tb, 0, st>>>(Y, n, m, sd, H, L, (int)ldk);
  SPB_LAUNCH_CHECK();
  CUtensorMap mH = make_map(H, m, (int)ldk, (int)ldk), mL = make_map(L, m, (int)ldk, (int)ldk);
  const size_t smem = (size_t)STAGES * STAGE_BYTES + 1024;
  SPB_CUDA(cudaFuncSetAttribute(gram_tile_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  gram_tile_kernel<<<(unsigned)ntiles, 128, smem, st>>>(mH, mL, tiles, m, (int)(ldk / BK), G, err);
  SPB_LAUNCH_CHECK();
  symmetrize_kernel<<<(unsigned)(((size_t)m * m + 255) / 256), 256, 0, st>>>(G, m, S);
  SPB_LAUNCH_CHECK();
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
