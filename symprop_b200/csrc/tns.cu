// Device-side ingest of the .tns text format read by the reference's
// SymtensLoader (src/utils/loader.cpp:8-36):
//     order dim
//     i1 i2 ... iN value        (one record per nonzero, 1-based ids)
// The loader reads whitespace-separated tokens with an std::istream, sorts
// each index tuple ascending and stops at the first read that fails or hits
// the end of the file (so a last value that ends the file with no trailing
// whitespace is dropped, as is a trailing partial record).
//
// Here the file's bytes are copied to the device once and tokenised there:
// token starts are selected from the byte stream (cub::DeviceSelect), then
// one thread parses one record (N unsigned integers and a double) and sorts
// its tuple.  Doubles take Clinger's exact fast path (W. D. Clinger, "How to
// read floating point numbers accurately", PLDI 1990): a decimal mantissa
// below 2^53 with a power of ten 10^k, |k| <= 22, is one correctly rounded
// IEEE multiplication or division of exact operands, so the result equals
// strtod's.  The few values outside it (more than 15-16 significant digits,
// or large exponents) are listed by the kernel and converted on the host
// with strtod, which the reference's stream extraction also uses.
#include <cub/cub.cuh>
#include <fcntl.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <thread>
#include <vector>

#include "common.cuh"
#include "tensor.cuh"

namespace spb {
namespace {

__host__ __device__ inline bool is_ws(char c) {
  return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r';
}

struct IsTokenStart {
  const char *b;
  __device__ bool operator()(uint32_t i) const { return !is_ws(b[i]) && (i == 0 || is_ws(b[i - 1])); }
};

// 10^0 .. 10^22 are exact doubles
__constant__ double kPow10[23] = {1e0,  1e1,  1e2,  1e3,  1e4,  1e5,  1e6,  1e7,  1e8,  1e9,  1e10, 1e11,
                                  1e12, 1e13, 1e14, 1e15, 1e16, 1e17, 1e18, 1e19, 1e20, 1e21, 1e22};

constexpr int kBadToken = 1, kBadRange = 2;
constexpr int kMaxTnsOrder = 8;  // the orders symprop_tensor_create accepts

// unsigned decimal integer token [+]digits (the ids are dim_t = uint32)
__device__ inline int parse_uint(const char *b, uint32_t s, uint32_t e, uint32_t &out) {
  if (s < e && b[s] == '+') ++s;
  if (s >= e) return kBadToken;
  uint64_t v = 0;
  for (uint32_t i = s; i < e; ++i) {
    const char c = b[i];
    if (c < '0' || c > '9') return kBadToken;
    v = v * 10 + (uint64_t)(c - '0');
    if (v > 0xffffffffull) return kBadRange;
  }
  out = (uint32_t)v;
  return 0;
}

// [+-] digits [. digits] [(e|E) [+-] digits], at least one mantissa digit.
// Returns 0 and the value when the fast path applies, -1 when the token is
// well formed but needs the host conversion, kBadToken otherwise.
__device__ inline int parse_double(const char *b, uint32_t s, uint32_t e, double &out) {
  bool neg = false;
  if (s < e && (b[s] == '+' || b[s] == '-')) neg = b[s++] == '-';
  uint64_t m = 0;
  int digits = 0, sig = 0, exp10 = 0;
  bool dropped = false;  // nonzero digits beyond 19 significant ones
  uint32_t i = s;
  for (; i < e && b[i] >= '0' && b[i] <= '9'; ++i, ++digits) {
    const int d = b[i] - '0';
    if (sig < 19) {
      if (m || d) { m = m * 10 + (uint64_t)d; ++sig; }
    } else {
      ++exp10;
      dropped |= d != 0;
    }
  }
  if (i < e && b[i] == '.') {
    for (++i; i < e && b[i] >= '0' && b[i] <= '9'; ++i, ++digits) {
      const int d = b[i] - '0';
      if (sig < 19) {
        if (m || d) { m = m * 10 + (uint64_t)d; ++sig; }
        --exp10;
      } else {
        dropped |= d != 0;
      }
    }
  }
  if (!digits) return kBadToken;
  if (i < e && (b[i] == 'e' || b[i] == 'E')) {
    ++i;
    bool eneg = false;
    if (i < e && (b[i] == '+' || b[i] == '-')) eneg = b[i++] == '-';
    if (i >= e) return kBadToken;
    int x = 0;
    for (; i < e && b[i] >= '0' && b[i] <= '9'; ++i) x = x < 100000 ? x * 10 + (b[i] - '0') : x;
    exp10 += eneg ? -x : x;
  }
  if (i != e) return kBadToken;
  if (m == 0 && !dropped) {
    out = neg ? -0.0 : 0.0;
    return 0;
  }
  if (dropped || m > (1ull << 53) || exp10 < -22 || exp10 > 22) return -1;
  const double v = (double)m;  // exact: m <= 2^53
  out = exp10 >= 0 ? v * kPow10[exp10] : v / kPow10[-exp10];
  if (neg) out = -out;
  return 0;
}

__device__ inline uint32_t token_end(const char *b, uint32_t s, uint32_t len) {
  while (s < len && !is_ws(b[s])) ++s;
  return s;
}

// One record per thread: N ids (sorted ascending) and the value.
__global__ void record_kernel(const char *b, uint32_t len, const uint32_t *starts, uint64_t nrec, uint32_t N,
                              uint32_t *inds, double *vals, unsigned long long *first_bad, int *bad_kind,
                              uint32_t *slow, unsigned long long *nslow) {
  const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nrec) return;
  const uint32_t *tk = starts + k * (N + 1);
  uint32_t id[kMaxTnsOrder];
  for (uint32_t f = 0; f < N; ++f) {
    const uint32_t s = tk[f];
    const int r = parse_uint(b, s, token_end(b, s, len), id[f]);
    if (r) {
      atomicMin(first_bad, (unsigned long long)k);
      atomicOr(bad_kind, r);
      return;
    }
  }
  // insertion sort of the tuple (std::sort in the loader)
  for (uint32_t a = 1; a < N; ++a) {
    const uint32_t x = id[a];
    uint32_t c = a;
    while (c > 0 && id[c - 1] > x) {
      id[c] = id[c - 1];
      --c;
    }
    id[c] = x;
  }
  for (uint32_t f = 0; f < N; ++f) inds[k * N + f] = id[f];
  const uint32_t s = tk[N];
  double v = 0.0;
  const int r = parse_double(b, s, token_end(b, s, len), v);
  if (r > 0) {
    atomicMin(first_bad, (unsigned long long)k);
    atomicOr(bad_kind, r);
    return;
  }
  if (r < 0) {
    const unsigned long long at = atomicAdd(nslow, 1ull);
    slow[at] = (uint32_t)k;
  }
  vals[k] = v;
}

__global__ void slow_offsets_kernel(const uint32_t *slow, uint64_t n, const uint32_t *starts, uint32_t N,
                                    uint32_t *off) {
  const uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) off[q] = starts[(uint64_t)slow[q] * (N + 1) + N];
}

__global__ void scatter_values_kernel(const uint32_t *slow, const double *v, uint64_t n, double *vals) {
  const uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) vals[slow[q]] = v[q];
}

inline unsigned grid_for(uint64_t n, unsigned block) {
  return (unsigned)std::max<uint64_t>(1, (n + block - 1) / block);
}

// header "order dim" read on the host (two tokens); returns the offset after it
uint64_t read_header(const char *b, uint64_t len, uint32_t &order, uint32_t &dim) {
  uint64_t i = 0;
  uint64_t val[2];
  for (int f = 0; f < 2; ++f) {
    while (i < len && is_ws(b[i])) ++i;
    uint64_t s = i;
    if (i < len && b[i] == '+') ++i;
    uint64_t v = 0;
    const uint64_t d0 = i;
    while (i < len && b[i] >= '0' && b[i] <= '9') {
      v = v * 10 + (uint64_t)(b[i] - '0');
      if (v > 0xffffffffull) fail(SYMPROP_ERR_INVALID, "tns header: value out of range at byte %llu",
                                  (unsigned long long)s);
      ++i;
    }
    if (i == d0 || (i < len && !is_ws(b[i])))
      fail(SYMPROP_ERR_INVALID, "tns header: expected 'order dim', malformed token at byte %llu",
           (unsigned long long)s);
    val[f] = v;
  }
  order = (uint32_t)val[0];
  dim = (uint32_t)val[1];
  return i;
}

}  // namespace

// Parses the file text into device arrays (sorted tuples, values).
void tns_parse_device(const char *h_bytes, uint64_t len, uint32_t &order, uint32_t &dim, uint64_t &nnz,
                      DBuf<uint32_t> &d_inds, DBuf<double> &d_vals) {
  NvtxRange nv("tns parse");
  const uint64_t body = read_header(h_bytes, len, order, dim);
  if (order < 2 || order > (uint32_t)kMaxTnsOrder)
    fail(SYMPROP_ERR_ORDER, "order %u not supported (2..%d)", order, kMaxTnsOrder);
  const uint64_t blen = len - body;
  if (blen >= 0xffffffffull) fail(SYMPROP_ERR_SIZE, "tns text above 4 GiB after the header");
  nnz = 0;
  if (blen == 0) return;
  cudaStream_t st = 0;
  const char *hb = h_bytes + body;
  DBuf<char> b(blen);
  SPB_CUDA(cudaMemcpy(b.p, hb, blen, cudaMemcpyHostToDevice));
  // token starts
  DBuf<uint32_t> starts(blen / 2 + 1);
  DBuf<uint64_t> ntok_d(1);
  {
    cub::CountingInputIterator<uint32_t> it(0);
    size_t tmp = 0;
    SPB_CUDA(cub::DeviceSelect::If(nullptr, tmp, it, starts.p, ntok_d.p, (uint32_t)blen, IsTokenStart{b.p}, st));
    DBuf<char> work(std::max<size_t>(tmp, 1));
    SPB_CUDA(cub::DeviceSelect::If(work.p, tmp, it, starts.p, ntok_d.p, (uint32_t)blen, IsTokenStart{b.p}, st));
  }
  uint64_t ntok = 0;
  SPB_CUDA(cudaMemcpy(&ntok, ntok_d.p, sizeof(uint64_t), cudaMemcpyDeviceToHost));
  const uint32_t N = order;
  uint64_t nrec = ntok / (N + 1);
  if (nrec && ntok % (N + 1) == 0) {
    // the last value ends the file with no trailing whitespace: the stream
    // hits end-of-file on it and the loader drops that record
    uint32_t last = 0;
    SPB_CUDA(cudaMemcpy(&last, starts.p + ntok - 1, sizeof(uint32_t), cudaMemcpyDeviceToHost));
    uint64_t e = last;
    while (e < blen && !is_ws(hb[e])) ++e;
    if (e == blen) --nrec;
  }
  if (nrec * (uint64_t)N >= (1ull << 32)) fail(SYMPROP_ERR_SIZE, "nnz*order must be below 2^32");
  d_inds.alloc(nrec * N);
  d_vals.alloc(nrec);
  if (!nrec) return;
  DBuf<unsigned long long> first_bad(1), nslow(1);
  DBuf<int> bad_kind(1);
  DBuf<uint32_t> slow(nrec);
  const unsigned long long none = ~0ull;
  SPB_CUDA(cudaMemcpy(first_bad.p, &none, sizeof(none), cudaMemcpyHostToDevice));
  SPB_CUDA(cudaMemset(nslow.p, 0, sizeof(unsigned long long)));
  SPB_CUDA(cudaMemset(bad_kind.p, 0, sizeof(int)));
  record_kernel<<<grid_for(nrec, 256), 256, 0, st>>>(b.p, (uint32_t)blen, starts.p, nrec, N, d_inds.p, d_vals.p,
                                                     first_bad.p, bad_kind.p, slow.p, nslow.p);
  SPB_LAUNCH_CHECK();
  unsigned long long hbad = 0, hslow = 0;
  int kind = 0;
  SPB_CUDA(cudaMemcpy(&hbad, first_bad.p, sizeof(hbad), cudaMemcpyDeviceToHost));
  SPB_CUDA(cudaMemcpy(&kind, bad_kind.p, sizeof(int), cudaMemcpyDeviceToHost));
  SPB_CUDA(cudaMemcpy(&hslow, nslow.p, sizeof(hslow), cudaMemcpyDeviceToHost));
  if (hbad != none) {
    uint32_t at = 0;
    SPB_CUDA(cudaMemcpy(&at, starts.p + hbad * (N + 1), sizeof(uint32_t), cudaMemcpyDeviceToHost));
    fail(SYMPROP_ERR_INVALID, "tns: %s in record %llu (line of the token at byte %llu)",
         (kind & kBadRange) ? "index above 2^32-1" : "malformed token", hbad + 1,
         (unsigned long long)(body + at));
  }
  if (hslow) {
    // values outside the exact fast path: strtod on the host (as the
    // stream does), all of them in one batch: token offsets down, values
    // up, one scatter
    DBuf<uint32_t> d_off(hslow);
    DBuf<double> d_fix(hslow);
    slow_offsets_kernel<<<grid_for(hslow, 256), 256, 0, st>>>(slow.p, hslow, starts.p, N, d_off.p);
    SPB_LAUNCH_CHECK();
    std::vector<uint32_t> off(hslow);
    std::vector<double> fixed(hslow);
    SPB_CUDA(cudaMemcpy(off.data(), d_off.p, hslow * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    const unsigned nth = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (unsigned w = 0; w < nth; ++w)
      pool.emplace_back([&, w] {
        char tok[512];
        for (size_t q = w; q < hslow; q += nth) {
          const uint64_t s0 = off[q];
          uint64_t e = s0;
          while (e < blen && !is_ws(hb[e])) ++e;
          const size_t l = (size_t)(e - s0);
          if (l < sizeof(tok)) {
            std::memcpy(tok, hb + s0, l);
            tok[l] = 0;
            fixed[q] = std::strtod(tok, nullptr);
          } else {
            fixed[q] = std::strtod(std::string(hb + s0, l).c_str(), nullptr);
          }
        }
      });
    for (auto &th : pool) th.join();
    SPB_CUDA(cudaMemcpy(d_fix.p, fixed.data(), hslow * sizeof(double), cudaMemcpyHostToDevice));
    scatter_values_kernel<<<grid_for(hslow, 256), 256, 0, st>>>(slow.p, d_fix.p, hslow, d_vals.p);
    SPB_LAUNCH_CHECK();
    SPB_CUDA(cudaDeviceSynchronize());
  }
  nnz = nrec;
}

// Reads `len` bytes of `path` from offset `off` into dst with up to 16
// threads, each taking 16 MiB pieces with pread: a file in the page cache
// then arrives at memory-copy speed rather than at one thread's.
static void read_parallel(const char *path, uint64_t off, uint64_t len, char *dst) {
  if (!len) return;
  const int fd = ::open(path, O_RDONLY);
  if (fd < 0) fail(SYMPROP_ERR_INVALID, "cannot open %s", path);
  const uint64_t piece = 16ull << 20, npieces = (len + piece - 1) / piece;
  const unsigned nth =
      (unsigned)std::min<uint64_t>(npieces, std::max(1u, std::min(16u, std::thread::hardware_concurrency())));
  std::atomic<uint64_t> next{0};
  std::atomic<bool> bad{false};
  auto work = [&] {
    for (uint64_t k; !bad && (k = next++) < npieces;) {
      const uint64_t a = k * piece, n = std::min(piece, len - a);
      for (uint64_t done = 0; done < n;) {
        const ssize_t r = ::pread(fd, dst + a + done, n - done, (off_t)(off + a + done));
        if (r <= 0) {
          bad = true;
          break;
        }
        done += (uint64_t)r;
      }
    }
  };
  std::vector<std::thread> pool;
  for (unsigned i = 1; i < nth; ++i) pool.emplace_back(work);
  work();
  for (auto &th : pool) th.join();
  ::close(fd);
  if (bad) fail(SYMPROP_ERR_INVALID, "short read of %s", path);
}

}  // namespace spb

using namespace spb;

extern "C" {

int symprop_tensor_load_tns(const char *path, symprop_tensor **out) {
  return guard([&] {
    if (!path || !out) fail(SYMPROP_ERR_INVALID, "null argument");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
      cudaGetLastError();
      fail(SYMPROP_ERR_NODEVICE, "no CUDA device visible");
    }
    std::FILE *f = std::fopen(path, "rb");
    if (!f) fail(SYMPROP_ERR_INVALID, "cannot open %s", path);
    std::fseek(f, 0, SEEK_END);
    const long sz = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    char *buf = nullptr;
    if (sz > 0 && cudaMallocHost(&buf, (size_t)sz) != cudaSuccess) {
      cudaGetLastError();
      std::fclose(f);
      fail(SYMPROP_ERR_OOM, "pinned host buffer of %ld bytes", sz);
    }
    std::unique_ptr<char, void (*)(char *)> hold(buf, [](char *p) { if (p) cudaFreeHost(p); });
    std::fclose(f);
    const size_t got = (size_t)std::max(sz, 0L);
    read_parallel(path, 0, got, buf);
    uint32_t order = 0, dim = 0;
    uint64_t nnz = 0;
    DBuf<uint32_t> inds;
    DBuf<double> vals;
    tns_parse_device(buf, (uint64_t)got, order, dim, nnz, inds, vals);
    if (dim == 0) fail(SYMPROP_ERR_INVALID, "dim must be positive");
    auto t = std::make_unique<symprop_tensor>();
    SPB_CUDA(cudaGetDevice(&t->s.device));
    t->s.order = order;
    t->s.dim = dim;
    t->s.nnz = nnz;
    tensor_build(t->s, inds.p, vals.p, true);
    *out = t.release();
  });
}

int symprop_tensor_load_spt(const char *path, symprop_tensor **out) {
  return guard([&] {
    if (!path || !out) fail(SYMPROP_ERR_INVALID, "null argument");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
      cudaGetLastError();
      fail(SYMPROP_ERR_NODEVICE, "no CUDA device visible");
    }
    std::FILE *f = std::fopen(path, "rb");
    if (!f) fail(SYMPROP_ERR_INVALID, "cannot open %s", path);
    std::unique_ptr<std::FILE, int (*)(std::FILE *)> fh(f, std::fclose);
    unsigned char head[24];
    if (std::fread(head, 1, sizeof head, f) != sizeof head || std::memcmp(head, "SPT1", 4) != 0)
      fail(SYMPROP_ERR_INVALID, "%s: not an SPT1 tuple file", path);
    uint32_t order = 0, dim = 0;
    uint64_t nnz = 0;
    std::memcpy(&order, head + 4, 4);
    std::memcpy(&dim, head + 8, 4);
    std::memcpy(&nnz, head + 16, 8);
    if (order < 2 || order > 8) fail(SYMPROP_ERR_ORDER, "order %u not supported (2..8)", order);
    if (dim == 0) fail(SYMPROP_ERR_INVALID, "dim must be positive");
    if (nnz >= (1ull << 32) / order) fail(SYMPROP_ERR_SIZE, "nnz*order must be below 2^32");
    std::fseek(f, 0, SEEK_END);
    const long sz = std::ftell(f);
    const uint64_t ibytes = nnz * order * 4, vbytes = nnz * 8;
    if (sz < 0 || (uint64_t)sz != sizeof head + ibytes + vbytes)
      fail(SYMPROP_ERR_INVALID, "%s: %ld bytes, the header announces %llu", path, sz,
           (unsigned long long)(sizeof head + ibytes + vbytes));
    std::fseek(f, (long)sizeof head, SEEK_SET);
    char *buf = nullptr;
    if (ibytes + vbytes && cudaMallocHost(&buf, ibytes + vbytes) != cudaSuccess) {
      cudaGetLastError();
      fail(SYMPROP_ERR_OOM, "pinned host buffer of %llu bytes", (unsigned long long)(ibytes + vbytes));
    }
    std::unique_ptr<char, void (*)(char *)> hold(buf, [](char *p) { if (p) cudaFreeHost(p); });
    read_parallel(path, sizeof head, ibytes + vbytes, buf);
    DBuf<uint32_t> inds(nnz * order);
    DBuf<double> vals(nnz);
    if (nnz) {
      SPB_CUDA(cudaMemcpy(inds.p, buf, ibytes, cudaMemcpyHostToDevice));
      SPB_CUDA(cudaMemcpy(vals.p, buf + ibytes, vbytes, cudaMemcpyHostToDevice));
    }
    auto t = std::make_unique<symprop_tensor>();
    SPB_CUDA(cudaGetDevice(&t->s.device));
    t->s.order = order;
    t->s.dim = dim;
    t->s.nnz = nnz;
    tensor_build(t->s, inds.p, vals.p, true);  // checks every id against [1, dim] and the tuple order
    *out = t.release();
  });
}

int symprop_tensor_save_spt(const symprop_tensor *t, const char *path) {
  return guard([&] {
    if (!t || !path) fail(SYMPROP_ERR_INVALID, "null argument");
    const uint32_t order = t->s.order, dim = t->s.dim, zero = 0;
    const uint64_t nnz = t->s.nnz;
    std::vector<uint32_t> inds(nnz * order);
    std::vector<double> vals(nnz);
    if (nnz && symprop_tensor_copy_nonzeros(t, inds.data(), vals.data()) != SYMPROP_OK)
      fail(SYMPROP_ERR_CUDA, "copying the nonzeros out failed");
    std::FILE *f = std::fopen(path, "wb");
    if (!f) fail(SYMPROP_ERR_INVALID, "cannot create %s", path);
    std::unique_ptr<std::FILE, int (*)(std::FILE *)> fh(f, std::fclose);
    bool ok = std::fwrite("SPT1", 1, 4, f) == 4 && std::fwrite(&order, 4, 1, f) == 1 &&
              std::fwrite(&dim, 4, 1, f) == 1 && std::fwrite(&zero, 4, 1, f) == 1 && std::fwrite(&nnz, 8, 1, f) == 1;
    if (ok && nnz)
      ok = std::fwrite(inds.data(), 4, inds.size(), f) == inds.size() &&
           std::fwrite(vals.data(), 8, vals.size(), f) == vals.size();
    if (!ok) fail(SYMPROP_ERR_INVALID, "short write of %s", path);
  });
}

int symprop_tensor_copy_nonzeros(const symprop_tensor *t, uint32_t *inds, double *vals) {
  return guard([&] {
    if (!t) fail(SYMPROP_ERR_INVALID, "null tensor");
    SPB_CUDA(cudaSetDevice(t->s.device));
    if (!t->s.nnz) return;
    if (inds) {  // stored 0-based on the device; the API is 1-based like the loader's
      const uint64_t cnt = t->s.nnz * t->s.order;
      SPB_CUDA(cudaMemcpy(inds, t->s.inds.p, cnt * sizeof(uint32_t), cudaMemcpyDeviceToHost));
      for (uint64_t i = 0; i < cnt; ++i) inds[i] += 1;
    }
    if (vals) SPB_CUDA(cudaMemcpy(vals, t->s.vals.p, t->s.nnz * sizeof(double), cudaMemcpyDeviceToHost));
  });
}

}  // extern "C"
