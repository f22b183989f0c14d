// s3ttmctc — drop-in for the reference's examples/s3ttmctc.cpp:
// `s3ttmctc <input_file> <R>` loads the .tns file, fills the factor
// (dim x R) from std::mt19937(1) through std::uniform_real_distribution(1.0,
// 2.0) (:55-61) and times ten rounds of the HOQRI inner step without the QR
// (:76-84): Y = S3TTMc(X, factor) packed, core = factor^T Y (gemmtn),
// factor = Y diag(coeff) core^T (symgemm).  Prints "Insertion time: X ms",
// one "S3TTMcTC Time: X ms" line per round and the FunctionTimer table,
// with the reference's usage / open-failure messages and exit codes.  The
// factor is not normalised between rounds, as in the reference, so its
// values grow with every round.  "Insertion time" here covers the device
// parse of the file and the tensor build.
#include <chrono>
#include <fstream>
#include <iostream>
#include <random>
#include <string>
#include <vector>

#include "symtucker.hpp"

using namespace symprop;

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
    const order_t order = symtens.order();
    std::vector<real_t> factor(dim * R);
    std::mt19937 gen(1);
    std::uniform_real_distribution<real_t> dist(1.0, 2.0);
    for (size_t i = 0; i < dim * R; i++) factor[i] = dist(gen);

    const size_t ncols = symtens_size(R, order - 1);
    std::vector<real_t> core(R * ncols);
    std::vector<real_t> Y(dim * ncols);
    const std::vector<real_t> coeff = symtens_coeff(R, order - 1);
    for (size_t i = 0; i < 10; i++) {
      t1 = std::chrono::high_resolution_clock::now();
      symtens.S3TTMc(Y, factor, (dim_t)R, true);
      matrix::gemmtn(core, factor, Y, dim, R, ncols);
      matrix::symgemm(factor, Y, core, coeff, dim, R);
      t2 = std::chrono::high_resolution_clock::now();
      std::cout << "S3TTMcTC Time: " << std::chrono::duration_cast<std::chrono::milliseconds>(t2 - t1).count()
                << " ms" << std::endl;
    }
    FunctionTimer::printTimes();
  } catch (const std::exception &e) {
    std::cerr << "s3ttmctc: " << e.what() << std::endl;
    return 1;
  }
  return 0;
}
