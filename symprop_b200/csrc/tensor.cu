// Tensor construction on the device: validation, ||X||, and the
// row-segmented owner list consumed by the S3TTMc kernels.
//
// Replaces the construction half of SpSymtensor::SpSymtensor
// (src/sparse/spsymtensor.cpp:16-28): the pointer trie insert
// (src/dtree.cpp:56-80) becomes one pass that emits, for every nonzero t and
// every distinct id e of t, the owner (row = e, leaf = t \ e) with
// coefficient f_e * v * mult(t)/N!, followed by a device radix sort of the
// owners by row.  calc_norm (src/sparse/spsymtensor.cpp:114-138) is a device
// reduction of v^2 * mult(t).
#include <cub/cub.cuh>

#include <algorithm>
#include <chrono>
#include <cstdlib>

#include "tensor.cuh"

namespace spb {

namespace {

constexpr int kMaxOrder = 16;

__global__ void iota_kernel(uint32_t *p, uint64_t n) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    p[i] = (uint32_t)i;
}

__global__ void validate_kernel(const uint32_t *inds, uint64_t nnz, uint32_t order,
                                uint32_t dim, uint32_t *inds0, int *bad) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nnz) return;
  const uint32_t *t = inds + i * order;
  uint32_t prev = 0;
  for (uint32_t j = 0; j < order; ++j) {
    uint32_t v = t[j];
    if (v < 1 || v > dim) { atomicOr(bad, 1); return; }
    if (j && v < prev) { atomicOr(bad, 2); return; }
    prev = v;
    inds0[i * order + j] = v - 1;
  }
}

// distinct ids per tuple and v^2 * mult(t)
__global__ void count_kernel(const uint32_t *inds0, const double *vals, uint64_t nnz,
                             uint32_t order, uint32_t *cnt, double *normsq) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nnz) return;
  const uint32_t *t = inds0 + i * order;
  uint32_t distinct = 1;
  uint64_t denom = 1, run = 1;
  for (uint32_t j = 1; j <= order; ++j) {
    if (j < order && t[j] == t[j - 1]) {
      ++run;
    } else {
      denom *= factorial_u64((int)run);
      run = 1;
      if (j < order) ++distinct;
    }
  }
  uint64_t mult = factorial_u64((int)order) / denom;  // multinomial_coeff
  cnt[i] = distinct;
  double v = vals[i];
  normsq[i] = v * v * (double)mult;
}

__global__ void emit_owners_kernel(const uint32_t *inds0, const double *vals, uint64_t nnz,
                                   uint32_t order, const uint32_t *off, uint32_t sstride,
                                   uint32_t *own_row, uint32_t *own_S, double *own_c) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nnz) return;
  uint32_t t[kMaxOrder];
  for (uint32_t j = 0; j < order; ++j) t[j] = inds0[i * order + j];
  uint64_t denom = 1, run = 1;
  for (uint32_t j = 1; j <= order; ++j) {
    if (j < order && t[j] == t[j - 1]) {
      ++run;
    } else {
      denom *= factorial_u64((int)run);
      run = 1;
    }
  }
  const uint64_t nfact = factorial_u64((int)order);
  // the reference's owner coefficient (src/compressed_dtree.cpp:493-503)
  const double coeff = vals[i] * (double)(nfact / denom) / (double)nfact;
  uint32_t o = off[i];
  uint32_t j = 0;
  while (j < order) {
    uint32_t e = j + 1;
    while (e < order && t[e] == t[j]) ++e;
    const uint32_t f = e - j;  // multiplicity of id t[j]
    own_row[o] = t[j];
    uint32_t *S = own_S + (uint64_t)o * sstride;
    uint32_t c = 0;
    for (uint32_t k = 0; k < order; ++k)
      if (k != j) S[c++] = t[k];
    for (; c < sstride; ++c) S[c] = 0;
    own_c[o] = (double)f * coeff;
    ++o;
    j = e;
  }
}

__global__ void gather_owners_kernel(const uint32_t *perm, uint64_t nown, uint32_t sstride,
                                     const uint32_t *S_in, const double *c_in,
                                     uint32_t *S_out, double *c_out, float *c32_out) {
  uint64_t o = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= nown) return;
  uint32_t src = perm[o];
  const uint4 *a = reinterpret_cast<const uint4 *>(S_in + (uint64_t)src * sstride);
  uint4 *b = reinterpret_cast<uint4 *>(S_out + o * sstride);
  for (uint32_t w = 0; w < sstride / 4; ++w) b[w] = a[w];
  double c = c_in[src];
  c_out[o] = c;
  c32_out[o] = (float)c;
}

__global__ void row_ptr_kernel(const uint32_t *rows_sorted, uint64_t nown, uint32_t dim,
                               uint64_t *row_ptr) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i > dim) return;
  uint64_t lo = 0, hi = nown;
  while (lo < hi) {
    uint64_t mid = (lo + hi) >> 1;
    if (rows_sorted[mid] < i) lo = mid + 1; else hi = mid;
  }
  row_ptr[i] = lo;
}

inline unsigned grid_for(uint64_t n, unsigned block) {
  return (unsigned)std::max<uint64_t>(1, (n + block - 1) / block);
}

}  // namespace

// The work items in row order: one chunk per row, rows with more than co
// owners cut into consecutive slices, each slice with its own partial-sum
// slot.  Returns the number of slots.
uint32_t cut_rows(const std::vector<uint64_t> &row_ptr, uint32_t dim, uint64_t co, std::vector<Chunk> &ch,
                  std::vector<SplitRow> &sp) {
  ch.clear();
  sp.clear();
  ch.reserve((size_t)dim + row_ptr[dim] / co + 1);
  uint32_t slot = 0;
  for (uint32_t i = 0; i < dim; ++i) {
    uint64_t b = row_ptr[i], e = row_ptr[(size_t)i + 1];
    uint64_t c = e - b;
    if (c <= co) {
      ch.push_back(Chunk{i, kDirect, b, e});
    } else {
      uint32_t s0 = slot;
      for (uint64_t x = b; x < e; x += co) ch.push_back(Chunk{i, slot++, x, std::min(e, x + co)});
      sp.push_back(SplitRow{i, s0, slot, 0});
    }
  }
  return slot;
}

static uint32_t row_order_items(const TensorState &t, std::vector<Chunk> &ch, std::vector<SplitRow> &sp) {
  return cut_rows(t.h_row_ptr, t.dim, t.chunk_owners, ch, sp);
}

// Stable sort of ch[b, e) by owner count, heaviest first: a counting sort,
// since no chunk holds more than max_owners owners.
void sort_heaviest_first(std::vector<Chunk> &ch, size_t b, size_t e, uint64_t max_owners) {
  std::vector<size_t> start(max_owners + 2, 0);
  for (size_t i = b; i < e; ++i) ++start[max_owners - (ch[i].oe - ch[i].ob) + 1];
  for (size_t k = 1; k < start.size(); ++k) start[k] += start[k - 1];
  std::vector<Chunk> out(e - b);
  for (size_t i = b; i < e; ++i) out[start[max_owners - (ch[i].oe - ch[i].ob)]++] = ch[i];
  std::copy(out.begin(), out.end(), ch.begin() + (std::ptrdiff_t)b);
}

void tensor_build(TensorState &t, const uint32_t *h_inds, const double *h_vals, bool on_device) {
  NvtxRange nv("tensor build");
  // SPB_TRACE_BUILD=1 prints the time of each phase (with a device sync)
  const bool trace = std::getenv("SPB_TRACE_BUILD") != nullptr;
  auto tlast = std::chrono::steady_clock::now();
  auto mark = [&](const char *phase) {
    if (!trace) return;
    SPB_CUDA(cudaDeviceSynchronize());
    const auto now = std::chrono::steady_clock::now();
    std::fprintf(stderr, "tensor build: %-28s %8.2f ms\n", phase,
                 std::chrono::duration<double, std::milli>(now - tlast).count());
    tlast = now;
  };
  const uint32_t N = t.order;
  const uint64_t nnz = t.nnz;
  cudaStream_t st = 0;
  if (N < 2 || N > (uint32_t)kMaxOrder) fail(SYMPROP_ERR_ORDER, "unsupported order %u", N);

  DBuf<uint32_t> raw(nnz * N);
  t.inds.alloc(nnz * N);
  t.vals.alloc(nnz);
  if (nnz) {
    const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    SPB_CUDA(cudaMemcpy(raw.p, h_inds, nnz * N * sizeof(uint32_t), kind));
    SPB_CUDA(cudaMemcpy(t.vals.p, h_vals, nnz * sizeof(double), kind));
  }
  mark("allocate + copy tuples in");
  DBuf<int> bad(1);
  SPB_CUDA(cudaMemset(bad.p, 0, sizeof(int)));
  if (nnz) {
    validate_kernel<<<grid_for(nnz, 256), 256, 0, st>>>(raw.p, nnz, N, t.dim, t.inds.p, bad.p);
    SPB_LAUNCH_CHECK();
  }
  int hbad = 0;
  SPB_CUDA(cudaMemcpy(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (hbad & 1) fail(SYMPROP_ERR_INVALID, "index out of range [1, %u]", t.dim);
  if (hbad & 2) fail(SYMPROP_ERR_INVALID, "index tuple not sorted ascending");
  raw.release();
  mark("validate");

  // owners per tuple + ||X||^2 terms
  DBuf<uint32_t> cnt(nnz + 1), off(nnz + 1);
  DBuf<double> normsq(nnz + 1);
  if (nnz) {
    count_kernel<<<grid_for(nnz, 256), 256, 0, st>>>(t.inds.p, t.vals.p, nnz, N, cnt.p, normsq.p);
    SPB_LAUNCH_CHECK();
  }
  SPB_CUDA(cudaMemset(cnt.p + nnz, 0, sizeof(uint32_t)));
  DBuf<double> dsum(1);
  {
    size_t tmp = 0;
    SPB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, cnt.p, off.p, nnz + 1, st));
    size_t tmp2 = 0;
    SPB_CUDA(cub::DeviceReduce::Sum(nullptr, tmp2, normsq.p, dsum.p, nnz, st));
    DBuf<char> work(std::max<size_t>(std::max(tmp, tmp2), 1));
    SPB_CUDA(cub::DeviceScan::ExclusiveSum(work.p, tmp, cnt.p, off.p, nnz + 1, st));
    if (nnz) {
      SPB_CUDA(cub::DeviceReduce::Sum(work.p, tmp2, normsq.p, dsum.p, nnz, st));
    } else {
      SPB_CUDA(cudaMemset(dsum.p, 0, sizeof(double)));
    }
  }
  uint32_t total = 0;
  double nsq = 0.0;
  SPB_CUDA(cudaMemcpy(&total, off.p + nnz, sizeof(uint32_t), cudaMemcpyDeviceToHost));
  SPB_CUDA(cudaMemcpy(&nsq, dsum.p, sizeof(double), cudaMemcpyDeviceToHost));
  t.norm = std::sqrt(nsq);
  mark("count owners, norm");
  t.nown = total;
  t.sstride = ((N - 1) + 3) / 4 * 4;
  if (N - 1 == 0) t.sstride = 4;

  DBuf<uint32_t> own_row(t.nown), S_tmp(t.nown * t.sstride);
  DBuf<double> c_tmp(t.nown);
  if (nnz) {
    emit_owners_kernel<<<grid_for(nnz, 128), 128, 0, st>>>(t.inds.p, t.vals.p, nnz, N, off.p,
                                                           t.sstride, own_row.p, S_tmp.p,
                                                           c_tmp.p);
    SPB_LAUNCH_CHECK();
  }
  cnt.release();
  off.release();
  normsq.release();
  mark("emit owners");

  // stable radix sort of owners by row
  DBuf<uint32_t> rows_sorted(t.nown), perm_in(t.nown), perm(t.nown);
  if (t.nown) {
    device_iota(perm_in.p, t.nown, st);
    int end_bit = bits_for(t.dim);
    size_t tmp = 0;
    SPB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, own_row.p, rows_sorted.p, perm_in.p,
                                             perm.p, t.nown, 0, end_bit, st));
    DBuf<char> work(std::max<size_t>(tmp, 1));
    SPB_CUDA(cub::DeviceRadixSort::SortPairs(work.p, tmp, own_row.p, rows_sorted.p, perm_in.p,
                                             perm.p, t.nown, 0, end_bit, st));
  }
  mark("sort owners by row");
  t.own_S.alloc(t.nown * t.sstride);
  t.own_c64.alloc(t.nown);
  t.own_c32.alloc(t.nown);
  if (t.nown) {
    gather_owners_kernel<<<grid_for(t.nown, 256), 256, 0, st>>>(perm.p, t.nown, t.sstride, S_tmp.p,
                                                                c_tmp.p, t.own_S.p, t.own_c64.p,
                                                                t.own_c32.p);
    SPB_LAUNCH_CHECK();
  }
  t.row_ptr.alloc((uint64_t)t.dim + 1);
  row_ptr_kernel<<<grid_for((uint64_t)t.dim + 1, 256), 256, 0, st>>>(rows_sorted.p, t.nown, t.dim,
                                                                     t.row_ptr.p);
  SPB_LAUNCH_CHECK();
  t.h_row_ptr.resize((size_t)t.dim + 1);
  SPB_CUDA(cudaMemcpy(t.h_row_ptr.data(), t.row_ptr.p, ((size_t)t.dim + 1) * sizeof(uint64_t),
                      cudaMemcpyDeviceToHost));
  mark("gather owners, row pointers");

  // Work items: rows with more than chunk_owners owners are cut into slices
  // whose partial sums a second kernel adds in a fixed order.
  const uint64_t target_items = 148ull * 8ull;
  uint64_t co = (t.nown + target_items - 1) / std::max<uint64_t>(target_items, 1);
  co = std::min<uint64_t>(std::max<uint64_t>(co, 16), 256);
  t.chunk_owners = (uint32_t)co;
  std::vector<Chunk> ch;
  std::vector<SplitRow> sp;
  const uint32_t slot = row_order_items(t, ch, sp);
  sort_heaviest_first(ch, 0, ch.size(), co);
  t.nchunks = (uint32_t)ch.size();
  t.nheavy = 0;
  while (t.nheavy < t.nchunks && ch[t.nheavy].oe - ch[t.nheavy].ob > kLightOwners) ++t.nheavy;
  t.nsplit = (uint32_t)sp.size();
  t.nslots = slot;
  t.chunks.alloc(ch.size());
  if (!ch.empty())
    SPB_CUDA(cudaMemcpy(t.chunks.p, ch.data(), ch.size() * sizeof(Chunk), cudaMemcpyHostToDevice));
  t.split.alloc(sp.size());
  if (!sp.empty())
    SPB_CUDA(cudaMemcpy(t.split.p, sp.data(), sp.size() * sizeof(SplitRow), cudaMemcpyHostToDevice));
  t.bands.clear();
  t.chain.reset();
  SPB_CUDA(cudaDeviceSynchronize());
  mark("work items (host) + upload");
}

void device_iota(uint32_t *p, uint64_t n, cudaStream_t st) {
  if (!n) return;
  iota_kernel<<<(unsigned)std::min<uint64_t>((n + 255) / 256, 148ull * 64), 256, 0, st>>>(p, n);
  SPB_LAUNCH_CHECK();
}

const RowBands &row_bands(TensorState &t, uint32_t nb) {
  nb = std::max<uint32_t>(1, std::min<uint32_t>(nb, std::max<uint32_t>(t.dim, 1)));
  auto found = t.bands.find(nb);
  if (found != t.bands.end()) return *found->second;
  auto b = std::make_unique<RowBands>();
  b->nb = nb;
  std::vector<Chunk> ch;
  std::vector<SplitRow> sp;
  row_order_items(t, ch, sp);
  b->row0.resize(nb + 1);
  b->chunk0.resize(nb + 1);
  b->split0.resize(nb + 1);
  for (uint32_t k = 0; k <= nb; ++k) {
    const uint32_t r = (uint32_t)((uint64_t)t.dim * k / nb);
    b->row0[k] = r;
    b->chunk0[k] = (uint32_t)(std::lower_bound(ch.begin(), ch.end(), r,
                                               [](const Chunk &c, uint32_t v) { return c.row < v; }) -
                              ch.begin());
    b->split0[k] = (uint32_t)(std::lower_bound(sp.begin(), sp.end(), r,
                                               [](const SplitRow &c, uint32_t v) { return c.row < v; }) -
                              sp.begin());
  }
  for (uint32_t k = 0; k < nb; ++k) sort_heaviest_first(ch, b->chunk0[k], b->chunk0[k + 1], t.chunk_owners);
  b->chunks.alloc(ch.size());
  if (!ch.empty())
    SPB_CUDA(cudaMemcpy(b->chunks.p, ch.data(), ch.size() * sizeof(Chunk), cudaMemcpyHostToDevice));
  b->split.alloc(sp.size());
  if (!sp.empty())
    SPB_CUDA(cudaMemcpy(b->split.p, sp.data(), sp.size() * sizeof(SplitRow), cudaMemcpyHostToDevice));
  return *(t.bands[nb] = std::move(b));
}

}  // namespace spb
