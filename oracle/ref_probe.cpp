// Test infrastructure only: a probe driver linked against the reference's own
// compiled sources (oracle/_ref).  It exposes what the reference computes on
// the S3TTMc path so that tests can compare the CUDA path with it:
//
//   ref_probe tree   <tensor.spt> <out.bin>                 CompressedDTree dump
//   ref_probe s3ttmc <tensor.spt> <R> <U.f64> <packed> <Y.f64>
//   ref_probe time   <tensor.spt> <R> <reps> <packed>       S3TTMc wall time
//   ref_probe load   <tensor.tns> <out.bin>                 SymtensLoader result
//                    (order u32, dim u32, nnz u64, ids, values) and its time
//
// <tensor.spt> is the binary tuple format written by symprop_b200 (magic
// "SPT1", order, dim, nnz, nnz*order uint32 1-based sorted ids, nnz float64).
// The tree dump reads the private members of the reference's
// CompressedDTree (include/detail/compressed_dtree.hpp:52-59), hence the
// access override below; nothing here modifies the reference.
#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <random>
#include <string>
#include <vector>
#include <memory>
#include <span>
#include <ranges>
#include <queue>
#include <unordered_map>
#include <map>
#include <mutex>

#define private public
#define protected public
#include <detail/sparse/spsymtensor.hpp>
#include <detail/compressed_dtree.hpp>
#undef private
#undef protected
#include <utils/loader.hpp>
#include <omp.h>

using namespace symprop;

struct Tuples {
  uint32_t order = 0, dim = 0;
  uint64_t nnz = 0;
  std::vector<dim_t> inds;
  std::vector<real_t> vals;
};

static Tuples read_spt(const char *path) {
  Tuples t;
  FILE *f = std::fopen(path, "rb");
  if (!f) { std::perror(path); std::exit(2); }
  char magic[4];
  uint32_t pad;
  if (std::fread(magic, 1, 4, f) != 4 || std::memcmp(magic, "SPT1", 4) != 0) {
    std::fprintf(stderr, "bad magic in %s\n", path); std::exit(2);
  }
  if (std::fread(&t.order, 4, 1, f) != 1 || std::fread(&t.dim, 4, 1, f) != 1 ||
      std::fread(&pad, 4, 1, f) != 1 || std::fread(&t.nnz, 8, 1, f) != 1) {
    std::fprintf(stderr, "short header\n"); std::exit(2);
  }
  t.inds.resize(t.nnz * t.order);
  t.vals.resize(t.nnz);
  if (std::fread(t.inds.data(), 4, t.inds.size(), f) != t.inds.size() ||
      std::fread(t.vals.data(), 8, t.vals.size(), f) != t.vals.size()) {
    std::fprintf(stderr, "short body\n"); std::exit(2);
  }
  std::fclose(f);
  return t;
}

template <class T> static void put(FILE *f, const T &v) { std::fwrite(&v, sizeof(T), 1, f); }
template <class T> static void putv(FILE *f, const std::vector<T> &v) {
  uint64_t n = v.size();
  put(f, n);
  if (n) std::fwrite(v.data(), sizeof(T), n, f);
}

int main(int argc, char **argv) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: ref_probe tree|s3ttmc|time ...\n");
    return 1;
  }
  std::string mode = argv[1];
  if (mode == "load" && argc >= 4) {
    auto l0 = std::chrono::steady_clock::now();
    SymtensLoader L(argv[2]);
    auto l1 = std::chrono::steady_clock::now();
    FILE *f = std::fopen(argv[3], "wb");
    uint32_t order = L.order(), dim = L.dim();
    uint64_t nnz = L.unnzs().size();
    put(f, order);
    put(f, dim);
    put(f, nnz);
    if (nnz) {
      std::fwrite(L.unnz_inds().data(), sizeof(dim_t), L.unnz_inds().size(), f);
      std::fwrite(L.unnzs().data(), sizeof(real_t), nnz, f);
    }
    std::fclose(f);
    std::printf("{\"load_ms\": %.3f, \"nnz\": %llu}\n",
                std::chrono::duration<double, std::milli>(l1 - l0).count(), (unsigned long long)nnz);
    return 0;
  }
  Tuples t = read_spt(argv[2]);
  auto t0 = std::chrono::steady_clock::now();
  SpSymtensor X(t.dim, t.order, t.inds, t.vals);
  auto t1 = std::chrono::steady_clock::now();
  double build_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();

  if (mode == "tree") {
    if (argc < 4) return 1;
    const CompressedDTree &cd = *X._cdtree;
    FILE *f = std::fopen(argv[3], "wb");
    put<uint32_t>(f, cd.depth);
    for (uint32_t l = 0; l < cd.depth; l++) {
      putv(f, cd.level_idx[l]);
      putv(f, cd.level_ptr[l]);
      putv(f, cd.dep_list[l]);
    }
    std::vector<uint64_t> rem;
    std::vector<double> val;
    for (auto &p : cd.nonzero) { rem.push_back(p.first); val.push_back(p.second); }
    putv(f, rem);
    putv(f, val);
    put<double>(f, X.norm());
    std::fclose(f);
    return 0;
  }
  if (mode == "s3ttmc") {
    if (argc < 7) return 1;
    dim_t R = std::atoi(argv[3]);
    bool packed = std::atoi(argv[5]) != 0;
    std::vector<real_t> U((size_t)t.dim * R);
    FILE *fu = std::fopen(argv[4], "rb");
    if (!fu || std::fread(U.data(), 8, U.size(), fu) != U.size()) { std::fprintf(stderr, "bad U\n"); return 2; }
    std::fclose(fu);
    size_t ncols = packed ? symtens_size(R, t.order - 1) : (size_t)std::pow(R, t.order - 1);
    std::vector<real_t> Y((size_t)t.dim * ncols);
    X.S3TTMc(Y, U, R, packed);
    FILE *fy = std::fopen(argv[6], "wb");
    std::fwrite(Y.data(), 8, Y.size(), fy);
    std::fclose(fy);
    return 0;
  }
  if (mode == "time") {
    if (argc < 6) return 1;
    dim_t R = std::atoi(argv[3]);
    int reps = std::atoi(argv[4]);
    bool packed = std::atoi(argv[5]) != 0;
    std::vector<real_t> U((size_t)t.dim * R);
    std::mt19937 gen(1);
    std::normal_distribution<real_t> dist(0.0, 1.0);
    for (auto &u : U) u = dist(gen);
    size_t ncols = packed ? symtens_size(R, t.order - 1) : (size_t)std::pow(R, t.order - 1);
    std::vector<real_t> Y((size_t)t.dim * ncols);
    std::vector<double> ms;
    for (int i = 0; i < reps; i++) {
      auto a = std::chrono::steady_clock::now();
      X.S3TTMc(Y, U, R, packed);
      auto b = std::chrono::steady_clock::now();
      ms.push_back(std::chrono::duration<double, std::milli>(b - a).count());
    }
    std::printf("{\"build_ms\": %.3f, \"threads\": %d, \"s3ttmc_ms\": [", build_ms,
                omp_get_max_threads());
    for (int i = 0; i < reps; i++) std::printf("%s%.3f", i ? ", " : "", ms[i]);
    std::printf("]}\n");
    return 0;
  }
  std::fprintf(stderr, "unknown mode %s\n", mode.c_str());
  return 1;
}
