// symtens_ttmc — drop-in for the reference's examples/symtens_ttmc.cpp:
// `symtens_ttmc <input_file> <R>` loads the .tns file, fills U (dim x R)
// from std::mt19937(1) through std::uniform_real_distribution(1.0, 2.0)
// (:53-59), runs one packed S3TTMc and writes every row of Y to ./ttmc.out
// in fixed notation with 5 decimals, each value followed by ", " and each
// row by a newline (:76-86).  Same stdout lines ("Insertion time: X ms",
// "S3TTMc Time: X ms") and the same usage / open-failure messages and exit
// codes.  "Insertion time" here covers the device parse of the file and the
// tensor build (the reference parses on the host before its timer starts).
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <random>
#include <string>
#include <thread>
#include <vector>

#include "symtucker.hpp"

using namespace symprop;

// Rows [r0, r1) of Y formatted as the reference's std::fixed,
// std::setprecision(5) stream writes them (that stream formats through the
// C library's "%.*f" in the "C" locale, as snprintf does here).
static std::string format_rows(const std::vector<real_t> &Y, size_t cols, size_t r0, size_t r1) {
  std::string s;
  s.reserve((r1 - r0) * cols * 12);
  char buf[512];
  for (size_t i = r0; i < r1; ++i) {
    for (size_t j = 0; j < cols; ++j) {
      const int k = std::snprintf(buf, sizeof buf, "%.5f, ", Y[i * cols + j]);
      s.append(buf, (size_t)std::min<int>(k, (int)sizeof buf - 1));
    }
    s.push_back('\n');
  }
  return s;
}

int main(int argc, char **argv) {
  if (argc < 3) {
    std::cerr << "Usage: " << argv[0] << " <input_file> <R>" << std::endl;
    return 1;
  }
  const std::string input_file = argv[1];
  const size_t R = std::stoi(argv[2]);  // as the reference: invalid text throws
  {
    std::ifstream probe(input_file);
    if (!probe.is_open()) {
      std::cerr << "Error opening file: " << input_file << std::endl;
      return 1;
    }
  }
  try {
    auto t1 = std::chrono::high_resolution_clock::now();
    SpSymtensor symtens = SpSymtensor::load(input_file);  // .tns text, or a binary SPT1 file
    auto t2 = std::chrono::high_resolution_clock::now();
    std::cout << "Insertion time: " << std::chrono::duration_cast<std::chrono::milliseconds>(t2 - t1).count()
              << " ms" << std::endl;

    const size_t dim = symtens.dim();
    std::vector<real_t> u_mat(dim * R);
    std::mt19937 gen(1);
    std::uniform_real_distribution<real_t> dist(1.0, 2.0);
    for (size_t i = 0; i < dim * R; i++) u_mat[i] = dist(gen);

    t1 = std::chrono::high_resolution_clock::now();
    const size_t cols = symtens_size((dim_t)R, symtens.order() - 1);
    std::vector<real_t> res(dim * cols);
    symtens.S3TTMc(res, u_mat, (dim_t)R, true);
    t2 = std::chrono::high_resolution_clock::now();
    std::cout << "S3TTMc Time: " << std::chrono::duration_cast<std::chrono::milliseconds>(t2 - t1).count()
              << " ms" << std::endl;

    // format row blocks on all host threads, write them in order
    const size_t nthreads = std::max<size_t>(1, std::min<size_t>(std::thread::hardware_concurrency(), 64));
    const size_t block = std::max<size_t>(1, std::min<size_t>(4096, (dim + nthreads - 1) / nthreads));
    std::ofstream out_file("ttmc.out", std::ios::binary);
    for (size_t b0 = 0; b0 < dim; b0 += block * nthreads) {
      std::vector<std::string> parts(nthreads);
      std::vector<std::thread> pool;
      for (size_t k = 0; k < nthreads; ++k) {
        const size_t r0 = std::min(dim, b0 + k * block), r1 = std::min(dim, r0 + block);
        if (r0 < r1) pool.emplace_back([&, k, r0, r1] { parts[k] = format_rows(res, cols, r0, r1); });
      }
      for (auto &th : pool) th.join();
      for (const auto &p : parts) out_file.write(p.data(), (std::streamsize)p.size());
    }
    out_file.close();
  } catch (const std::exception &e) {
    std::cerr << "symtens_ttmc: " << e.what() << std::endl;
    return 1;
  }
  return 0;
}
