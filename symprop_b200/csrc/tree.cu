// Device construction of the reference's CompressedDTree arrays.
//
// Replaces DTree::banerjee_insert (src/dtree.cpp:38-80),
// CompressedDTree::CompressedDTree (src/compressed_dtree.cpp:13-90) and
// init_dep_list (:92-131).  The pointer trie is never built:
//  * level l (0-based) of the trie is the set of sorted (l+1)-sub-multisets
//    of the tuples, listed in lexicographic order (the BFS of a trie whose
//    children are visited in ascending id order).  Each tuple emits all its
//    C(N, l+1) position subsets as packed keys; a device LSD radix sort
//    (CUB, one pass per 64-bit key word) and a unique pass give the level;
//  * level_ptr[l] (children CSR) comes from each child's prefix, found by a
//    device binary search in level l;
//  * dep_list[l][j*(l+1)+k] = index in level l-1 of node j without its k-th
//    id, by binary search;
//  * the leaf level is generated in the reference's insertion order (nonzero
//    ascending, removed position N-1 down to 0, src/dtree.cpp:64-79) and
//    stably sorted, so the segment starts of the sorted keys are the owner
//    CSR and the owners appear in the reference's order.
// Keys pack E = floor(64/b) ids of b = bits(dim) bits per 64-bit word, first
// id in the most significant bits, so word-wise comparison is
// lexicographic order.
#include <cub/cub.cuh>


#include "tensor.cuh"

namespace spb {
namespace {

constexpr int kMaxWords = 4;

struct KeyFmt {
  int b = 0, E = 0, len = 0, words = 0;
};

KeyFmt key_fmt(uint32_t dim, int len) {
  KeyFmt f;
  f.b = bits_for(dim);
  f.E = 64 / f.b;
  f.len = len;
  f.words = (len + f.E - 1) / f.E;
  if (f.words > kMaxWords)
    fail(SYMPROP_ERR_SIZE, "tree keys of %d ids x %d bits exceed %d words", len, f.b, kMaxWords);
  return f;
}

__device__ __forceinline__ void pack_key(const uint32_t *ids, int len, int b, int E, int words,
                                         uint64_t *out) {
  for (int w = 0; w < words; ++w) out[w] = 0;
  for (int i = 0; i < len; ++i) {
    int w = i / E, s = (E - 1 - (i - w * E)) * b;
    out[w] |= (uint64_t)ids[i] << s;
  }
}

__device__ __forceinline__ uint32_t key_elem(const uint64_t *key, int i, int b, int E) {
  int w = i / E, s = (E - 1 - (i - w * E)) * b;
  return (uint32_t)((key[w] >> s) & ((1ull << b) - 1));
}

// keys of all position subsets `masks` (popcount len) of every tuple,
// word-major: words[w * cnt + item]
__global__ void gen_keys_kernel(const uint32_t *inds0, uint64_t nnz, uint32_t order,
                                const uint32_t *masks, uint32_t nmask, KeyFmt f, uint64_t *words,
                                uint64_t cnt) {
  uint64_t item = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (item >= cnt) return;
  uint64_t i = item / nmask;
  uint32_t mk = masks[item - i * nmask];
  uint32_t ids[16];
  int c = 0;
  for (uint32_t k = 0; k < order; ++k)
    if (mk & (1u << k)) ids[c++] = inds0[i * order + k] + 1;  // 1-based like the reference
  uint64_t key[kMaxWords];
  pack_key(ids, c, f.b, f.E, f.words, key);
  for (int w = 0; w < f.words; ++w) words[(uint64_t)w * cnt + item] = key[w];
}

__global__ void gather_word_kernel(const uint64_t *src, const uint32_t *perm, uint64_t cnt,
                                   uint64_t *dst) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < cnt) dst[i] = src[perm[i]];
}

__global__ void flag_new_kernel(const uint64_t *words, const uint32_t *perm, uint64_t cnt,
                                int nw, uint32_t *flag) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= cnt) return;
  uint32_t f = 1;
  if (i > 0) {
    f = 0;
    for (int w = 0; w < nw; ++w)
      if (words[(uint64_t)w * cnt + perm[i]] != words[(uint64_t)w * cnt + perm[i - 1]]) f = 1;
  }
  flag[i] = f;
}

// scatter unique keys (node-major) and, for the leaf level, segment starts
__global__ void compact_kernel(const uint64_t *words, const uint32_t *perm, const uint32_t *flag,
                               const uint32_t *pos, uint64_t cnt, int nw, uint64_t *nodes,
                               uint64_t *seg_start) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= cnt || !flag[i]) return;
  uint32_t u = pos[i];
  for (int w = 0; w < nw; ++w) nodes[(uint64_t)u * nw + w] = words[(uint64_t)w * cnt + perm[i]];
  if (seg_start) seg_start[u] = i;
}

__global__ void last_id_kernel(const uint64_t *nodes, uint64_t n, KeyFmt f, uint32_t *idx) {
  uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j < n) idx[j] = key_elem(nodes + j * f.words, f.len - 1, f.b, f.E);
}

// (N-1)! / prod(freq!) of each leaf multiset
__global__ void leaf_mult_kernel(const uint64_t *nodes, uint64_t n, KeyFmt f, double *out) {
  uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  uint64_t denom = 1, run = 1;
  uint32_t prev = key_elem(nodes + j * f.words, 0, f.b, f.E);
  for (int i = 1; i <= f.len; ++i) {
    uint32_t x = i < f.len ? key_elem(nodes + j * f.words, i, f.b, f.E) : 0xffffffffu;
    if (i < f.len && x == prev) {
      ++run;
    } else {
      denom *= factorial_u64((int)run);
      run = 1;
    }
    prev = x;
  }
  out[j] = (double)(factorial_u64(f.len) / denom);
}

__device__ int cmp_key(const uint64_t *a, const uint64_t *b, int nw) {
  for (int w = 0; w < nw; ++w)
    if (a[w] != b[w]) return a[w] < b[w] ? -1 : 1;
  return 0;
}

// dep_list: node j of level l (fmt f) without id k, searched in level l-1 (fmt g)
__global__ void dep_kernel(const uint64_t *nodes, uint64_t n, KeyFmt f, const uint64_t *prev,
                           uint64_t nprev, KeyFmt g, uint64_t *dep, int *missing) {
  uint64_t item = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (item >= n * (uint64_t)f.len) return;
  uint64_t j = item / f.len;
  int k = (int)(item - j * f.len);
  uint32_t ids[16];
  int c = 0;
  for (int i = 0; i < f.len; ++i)
    if (i != k) ids[c++] = key_elem(nodes + j * f.words, i, f.b, f.E);
  uint64_t key[kMaxWords];
  pack_key(ids, c, g.b, g.E, g.words, key);
  uint64_t lo = 0, hi = nprev;
  while (lo < hi) {
    uint64_t mid = (lo + hi) >> 1;
    if (cmp_key(prev + mid * g.words, key, g.words) < 0) lo = mid + 1; else hi = mid;
  }
  if (lo >= nprev || cmp_key(prev + lo * g.words, key, g.words) != 0) atomicOr(missing, 1);
  dep[item] = lo;
}

// level_ptr[l][j] = first child whose parent index >= j
__global__ void child_ptr_kernel(const uint64_t *dep_child, uint64_t nchild, int child_len,
                                 uint64_t nparent, uint64_t *ptr) {
  uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j > nparent) return;
  uint64_t lo = 0, hi = nchild;
  while (lo < hi) {
    uint64_t mid = (lo + hi) >> 1;
    uint64_t par = dep_child[mid * child_len + (child_len - 1)];
    if (par < j) lo = mid + 1; else hi = mid;
  }
  ptr[j] = lo;
}

__global__ void owners_kernel(const uint32_t *perm, uint64_t nown, const uint32_t *inds0,
                              const double *vals, uint32_t order, uint64_t *rem, double *val) {
  uint64_t x = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= nown) return;
  uint64_t e = perm[x];
  uint64_t i = e / order;
  uint32_t j = order - 1 - (uint32_t)(e - i * order);
  rem[x] = (uint64_t)inds0[i * order + j] + 1;
  val[x] = vals[i];
}

inline unsigned grid(uint64_t n, unsigned b = 256) {
  return (unsigned)std::max<uint64_t>(1, (n + b - 1) / b);
}

// Sorts `cnt` keys (word-major in `words`) lexicographically, stably;
// returns the permutation, unique node keys (node-major) and, optionally,
// the sorted position of each unique key's first occurrence.
uint64_t sort_unique(DBuf<uint64_t> &words, uint64_t cnt, const KeyFmt &f, DBuf<uint32_t> &perm,
                     DBuf<uint64_t> &nodes, DBuf<uint64_t> *seg_start) {
  cudaStream_t st = 0;
  perm.alloc(cnt);
  device_iota(perm.p, cnt, st);
  DBuf<uint64_t> kin(cnt), kout(cnt);
  DBuf<uint32_t> pout(cnt);
  size_t tmp = 0;
  if (cnt)
    SPB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, kin.p, kout.p, perm.p, pout.p, cnt, 0,
                                             64, st));
  DBuf<char> work(std::max<size_t>(tmp, 1));
  const int endbit = std::min(64, f.E * f.b);
  for (int w = f.words - 1; w >= 0 && cnt; --w) {
    gather_word_kernel<<<grid(cnt), 256, 0, st>>>(words.p + (uint64_t)w * cnt, perm.p, cnt, kin.p);
    SPB_LAUNCH_CHECK();
    SPB_CUDA(cub::DeviceRadixSort::SortPairs(work.p, tmp, kin.p, kout.p, perm.p, pout.p, cnt, 0,
                                             endbit, st));
    std::swap(perm.p, pout.p);
  }
  kin.release();
  kout.release();
  DBuf<uint32_t> flag(cnt + 1), pos(cnt + 1);
  if (cnt) {
    flag_new_kernel<<<grid(cnt), 256, 0, st>>>(words.p, perm.p, cnt, f.words, flag.p);
    SPB_LAUNCH_CHECK();
  }
  SPB_CUDA(cudaMemset(flag.p + cnt, 0, 4));
  size_t tmp2 = 0;
  SPB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp2, flag.p, pos.p, cnt + 1, st));
  work.ensure(std::max<size_t>(tmp2, 1));
  SPB_CUDA(cub::DeviceScan::ExclusiveSum(work.p, tmp2, flag.p, pos.p, cnt + 1, st));
  uint32_t nu = 0;
  SPB_CUDA(cudaMemcpy(&nu, pos.p + cnt, 4, cudaMemcpyDeviceToHost));
  nodes.alloc((uint64_t)nu * f.words);
  if (seg_start) seg_start->alloc((uint64_t)nu + 1);
  if (cnt) {
    compact_kernel<<<grid(cnt), 256, 0, st>>>(words.p, perm.p, flag.p, pos.p, cnt, f.words, nodes.p,
                                              seg_start ? seg_start->p : nullptr);
    SPB_LAUNCH_CHECK();
  }
  if (seg_start) SPB_CUDA(cudaMemcpy(seg_start->p + nu, &cnt, 8, cudaMemcpyHostToDevice));
  return nu;
}

}  // namespace

void tree_build(TensorState &t) {
  NvtxRange nv("CompressedDTree");
  if (t.tree) return;
  const uint32_t N = t.order;
  if (N < 2) fail(SYMPROP_ERR_ORDER, "order %u has no tree", N);
  if (t.nnz * (uint64_t)N >= (1ull << 32)) fail(SYMPROP_ERR_SIZE, "too many owners for the tree export");
  auto tr = std::make_unique<TreeLevels>();
  const uint32_t depth = N - 1;
  tr->depth = depth;
  tr->size.assign(depth, 0);
  tr->level_idx.resize(depth);
  tr->level_ptr.resize(depth);
  tr->dep_list.resize(depth);
  std::vector<DBuf<uint64_t>> nodes(depth);
  std::vector<KeyFmt> fmt(depth);
  cudaStream_t st = 0;

  for (uint32_t l = 0; l < depth; ++l) {
    const int len = (int)l + 1;
    fmt[l] = key_fmt(t.dim, len);
    const KeyFmt &f = fmt[l];
    std::vector<uint32_t> masks;
    if (l + 1 == depth) {
      // leaf level in insertion order: removed position j = N-1 .. 0
      for (int j = (int)N - 1; j >= 0; --j) masks.push_back(((1u << N) - 1) & ~(1u << j));
    } else {
      for (uint32_t mk = 0; mk < (1u << N); ++mk)
        if ((uint32_t)__builtin_popcount(mk) == (uint32_t)len) masks.push_back(mk);
    }
    DBuf<uint32_t> dmasks(masks.size());
    SPB_CUDA(cudaMemcpy(dmasks.p, masks.data(), masks.size() * 4, cudaMemcpyHostToDevice));
    const uint64_t cnt = t.nnz * masks.size();
    if (cnt >= (1ull << 32)) fail(SYMPROP_ERR_SIZE, "tree level %u has too many sub-multisets", l);
    DBuf<uint64_t> words(cnt * f.words);
    if (cnt) {
      gen_keys_kernel<<<grid(cnt), 256, 0, st>>>(t.inds.p, t.nnz, N, dmasks.p, (uint32_t)masks.size(),
                                                 f, words.p, cnt);
      SPB_LAUNCH_CHECK();
    }
    DBuf<uint32_t> perm;
    if (l + 1 == depth) {
      DBuf<uint64_t> seg;
      uint64_t nu = sort_unique(words, cnt, f, perm, nodes[l], &seg);
      tr->size[l] = nu;
      tr->level_ptr[l] = std::move(seg);  // owner CSR
      tr->nown = cnt;
      tr->own_rem.alloc(cnt);
      tr->own_val.alloc(cnt);
      if (cnt) {
        owners_kernel<<<grid(cnt), 256, 0, st>>>(perm.p, cnt, t.inds.p, t.vals.p, N, tr->own_rem.p,
                                                 tr->own_val.p);
        SPB_LAUNCH_CHECK();
      }
      tr->leaf_mult.alloc(std::max<uint64_t>(nu, 1));
      if (nu) {
        leaf_mult_kernel<<<grid(nu), 256, 0, st>>>(nodes[l].p, nu, f, tr->leaf_mult.p);
        SPB_LAUNCH_CHECK();
      }
    } else {
      tr->size[l] = sort_unique(words, cnt, f, perm, nodes[l], nullptr);
    }
    tr->level_idx[l].alloc(std::max<uint64_t>(tr->size[l], 1));
    if (tr->size[l]) {
      last_id_kernel<<<grid(tr->size[l]), 256, 0, st>>>(nodes[l].p, tr->size[l], f,
                                                        tr->level_idx[l].p);
      SPB_LAUNCH_CHECK();
    }
  }
  DBuf<int> missing(1);
  SPB_CUDA(cudaMemset(missing.p, 0, sizeof(int)));
  for (uint32_t l = 1; l < depth; ++l) {
    const uint64_t n = tr->size[l];
    tr->dep_list[l].alloc(std::max<uint64_t>(n * (l + 1), 1));
    if (n) {
      dep_kernel<<<grid(n * (l + 1)), 256, 0, st>>>(nodes[l].p, n, fmt[l], nodes[l - 1].p,
                                                    tr->size[l - 1], fmt[l - 1],
                                                    tr->dep_list[l].p, missing.p);
      SPB_LAUNCH_CHECK();
    }
  }
  for (uint32_t l = 0; l + 1 < depth; ++l) {
    tr->level_ptr[l].alloc(tr->size[l] + 1);
    child_ptr_kernel<<<grid(tr->size[l] + 1), 256, 0, st>>>(tr->dep_list[l + 1].p, tr->size[l + 1],
                                                           (int)l + 2, tr->size[l],
                                                           tr->level_ptr[l].p);
    SPB_LAUNCH_CHECK();
  }
  int hmiss = 0;
  SPB_CUDA(cudaMemcpy(&hmiss, missing.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (hmiss) fail(SYMPROP_ERR_INVALID, "tree build: a sub-multiset is missing from its level");
  SPB_CUDA(cudaDeviceSynchronize());
  t.tree = std::move(tr);
}

}  // namespace spb
