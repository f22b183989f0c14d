// symtucker — drop-in CLI for the reference's examples/symtucker.cpp:
// same flags (-f -r -i -t -d -a -s -o -init -h, parse at :43-84), same
// stdout lines ("Insertion time", "Running <ALG> algorithm", per-iteration
// lines, "---------- Time: X ms ----------", the timer table) and the same
// -o output format (SymTuckerDecomp::print).  Additional flags of the B200
// build: -p fp64|mixed (precision; default fp64 = the reference's FP64
// arithmetic), -q (suppress per-iteration lines).  "Insertion time" covers
// the device parse of the file and the tensor build (the reference parses
// on the host before its timer starts).  -f also takes a binary SPT1 tuple
// file (symprop_tensor_load_spt), recognised by its first four bytes.
#include <chrono>
#include <cstring>
#include <fstream>
#include <iostream>
#include <optional>
#include <string>

#include "symtucker.hpp"

using namespace symprop;

template <typename Alg>
static SymTuckerDecomp run_algorithm(Alg alg, const Config &con, const std::string &name) {
  std::cout << "Running " << name << " algorithm" << std::endl;
  auto t1 = std::chrono::high_resolution_clock::now();
  auto tucker = alg(con);
  auto t2 = std::chrono::high_resolution_clock::now();
  auto duration = std::chrono::duration_cast<std::chrono::milliseconds>(t2 - t1).count();
  std::cout << "---------- Time: " << duration << " ms ----------" << std::endl;
  FunctionTimer::printTimes();
  FunctionTimer::clear();
  return tucker;
}

static void help(const char *prog) {
  std::cout << prog
            << " -f <input_file> -i <max_iter> -r <rank> -t <rel_tol> -d "
               "<delta> -a <alg> -s <seed> -o <output_file> -init <init method>"
            << std::endl;
}

struct Input {
  Config config;
  std::string filePath;
  std::string outputFile;
  int alg = -1;
};

static std::optional<Input> parse(int argc, char **argv) {
  Input input;
  for (int i = 1; i < argc; i++) {
    std::string arg = argv[i];
    if (arg == "-f" && i + 1 < argc) {
      input.filePath = argv[++i];
    } else if (arg == "-i" && i + 1 < argc) {
      input.config.max_iter = (index_t)std::stod(argv[++i]);
    } else if (arg == "-r" && i + 1 < argc) {
      input.config.rank = std::stoi(argv[++i]);
    } else if (arg == "-t" && i + 1 < argc) {
      input.config.rel_tol = std::stod(argv[++i]);
    } else if (arg == "-d" && i + 1 < argc) {
      input.config.delta = std::stod(argv[++i]);
    } else if (arg == "-a" && i + 1 < argc) {
      input.alg = std::stoi(argv[++i]);
    } else if (arg == "-s" && i + 1 < argc) {
      input.config.seed = std::stoi(argv[++i]);
    } else if (arg == "-o" && i + 1 < argc) {
      input.outputFile = argv[++i];
    } else if (arg == "-init" && i + 1 < argc) {
      input.config.init = argv[++i];
    } else if (arg == "-p" && i + 1 < argc) {
      std::string p = argv[++i];
      input.config.precision = (p == "mixed") ? SYMPROP_PREC_MIXED : SYMPROP_PREC_FP64;
    } else if (arg == "-q") {
      input.config.verbose = false;
    } else if (arg == "-h") {
      help(argv[0]);
      return std::nullopt;
    } else {
      std::cout << "Option " << argv[i] << " is not defined\n";
      help(argv[0]);
      return std::nullopt;
    }
  }
  return input;
}

int main(int argc, char **argv) {
  auto input = parse(argc, argv);
  if (!input.has_value()) return 1;
  try {
    // The .tns text is parsed on the device (SpSymtensor::load_tns, the same
    // tensor as SymtensLoader + SpSymtensor for every file the reference
    // reads completely).  Text the device parser rejects, such as a token the
    // reference's stream reads only in part, and an unreadable file go
    // through SymtensLoader, whose stream semantics and messages decide.
    auto t1 = std::chrono::high_resolution_clock::now();
    std::optional<SpSymtensor> loaded;
    if (SpSymtensor::is_spt(input->filePath)) {  // binary SPT1 tuple file: no text rules apply
      loaded.emplace(SpSymtensor::load_spt(input->filePath));
    } else if (std::ifstream(input->filePath).is_open()) {
      try {
        loaded.emplace(SpSymtensor::load_tns(input->filePath));
      } catch (const std::runtime_error &) {
      }
    }
    if (!loaded) {
      SymtensLoader loader(input->filePath);
      t1 = std::chrono::high_resolution_clock::now();
      loaded.emplace(loader.dim(), loader.order(), loader.unnz_inds(), loader.unnzs());
    }
    SpSymtensor &symtens = *loaded;
    auto t2 = std::chrono::high_resolution_clock::now();
    auto duration = std::chrono::duration_cast<std::chrono::milliseconds>(t2 - t1).count();
    std::cout << "Insertion time: " << duration << " ms" << std::endl;
    FunctionTimer::printTimes();
    FunctionTimer::clear();

    std::string outpath = input->outputFile;
    if (outpath.empty()) outpath = "/dev/null";
    else if (outpath == "stdout") outpath = "/dev/stdout";
    else if (outpath == "stderr") outpath = "/dev/stderr";
    std::ofstream out(outpath);

    auto hooi = [&symtens](const Config &c) { return symtens.TuckerHOOI(c); };
    auto hoqri = [&symtens](const Config &c) { return symtens.TuckerHOQRI(c); };
    auto alt = [&symtens](const Config &c) { return symtens.TuckerAltHOOI(c); };
    if (input->alg == -1) {
      run_algorithm(hooi, input->config, "HOOI").print(out);
      run_algorithm(hoqri, input->config, "HOQRI").print(out);
      run_algorithm(alt, input->config, "AltHOOI").print(out);
      return 0;
    } else if (input->alg == 0) {
      run_algorithm(hooi, input->config, "HOOI").print(out);
    } else if (input->alg == 1) {
      run_algorithm(hoqri, input->config, "HOQRI").print(out);
    } else if (input->alg == 2) {
      run_algorithm(alt, input->config, "AltHOOI").print(out);
    }
  } catch (const std::exception &e) {
    std::cerr << "symtucker: " << e.what() << std::endl;
    return 2;
  }
  return 0;
}
