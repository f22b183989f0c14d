// symtucker: command-line front end of the B200 Tucker path, a drop-in for
// the reference's examples/symtucker.cpp.  What a caller can observe is kept:
//   * the flags -f -r -i -t -d -a -s -o -init -h and how each value is
//     converted (-i, -t, -d through std::stod; -r, -a, -s through std::stoi);
//   * an unknown flag, or a flag whose value is missing, prints
//     "Option <flag> is not defined" and the usage line and exits 1;
//   * the stdout lines "Insertion time: X ms", "Running <ALG> algorithm",
//     the per-iteration lines, "---------- Time: X ms ----------" and the
//     function-timer table;
//   * -a -1 (the default) runs HOOI, HOQRI and AltHOOI in that order, 0/1/2
//     one of them, any other value none;
//   * -o names a file, "stdout" or "stderr"; without it the factors go to
//     /dev/null.
// Flags of the B200 build: -p fp64|mixed (arithmetic; fp64, the default, is
// the reference's) and -q (no per-iteration lines).  "Insertion time" here
// covers the device parse and the tensor build.  -f also takes a binary
// SPT1 tuple file, recognised by its first four bytes.
#include <array>
#include <chrono>
#include <fstream>
#include <iostream>
#include <optional>
#include <string>
#include <string_view>

#include "symtucker.hpp"

using namespace symprop;

namespace {

using Clock = std::chrono::high_resolution_clock;

long long elapsed_ms(Clock::time_point since) {
  return std::chrono::duration_cast<std::chrono::milliseconds>(Clock::now() - since).count();
}

// What the command line asks for.
struct Request {
  Config cfg;
  std::string tensor_path;
  std::string factor_sink;  // -o value as given ("" = none)
  int which = -1;           // -a: -1 = all three
};

// One entry per flag: its spelling and how its value lands in the request.
// `apply` is null for the flags that take no value.
struct FlagRule {
  std::string_view flag;
  void (*apply)(Request &, const std::string &);
};

constexpr std::array<FlagRule, 11> kRules{{
    {"-f", [](Request &q, const std::string &v) { q.tensor_path = v; }},
    {"-i", [](Request &q, const std::string &v) { q.cfg.max_iter = (index_t)std::stod(v); }},
    {"-r", [](Request &q, const std::string &v) { q.cfg.rank = std::stoi(v); }},
    {"-t", [](Request &q, const std::string &v) { q.cfg.rel_tol = std::stod(v); }},
    {"-d", [](Request &q, const std::string &v) { q.cfg.delta = std::stod(v); }},
    {"-a", [](Request &q, const std::string &v) { q.which = std::stoi(v); }},
    {"-s", [](Request &q, const std::string &v) { q.cfg.seed = std::stoi(v); }},
    {"-o", [](Request &q, const std::string &v) { q.factor_sink = v; }},
    {"-init", [](Request &q, const std::string &v) { q.cfg.init = v; }},
    {"-p",
     [](Request &q, const std::string &v) {
       q.cfg.precision = v == "mixed" ? SYMPROP_PREC_MIXED : SYMPROP_PREC_FP64;
     }},
    {"-q", nullptr},
}};

void usage(const char *prog) {
  std::cout << prog
            << " -f <input_file> -i <max_iter> -r <rank> -t <rel_tol> -d "
               "<delta> -a <alg> -s <seed> -o <output_file> -init <init method>"
            << std::endl;
}

// The request, or nothing when the program should stop (help or a bad flag).
std::optional<Request> read_command_line(int argc, char **argv) {
  Request q;
  int i = 1;
  while (i < argc) {
    const std::string word = argv[i];
    if (word == "-h") {
      usage(argv[0]);
      return std::nullopt;
    }
    const FlagRule *rule = nullptr;
    for (const FlagRule &r : kRules)
      if (r.flag == word) rule = &r;
    const bool needs_value = rule && rule->apply;
    if (!rule || (needs_value && i + 1 >= argc)) {
      std::cout << "Option " << word << " is not defined\n";
      usage(argv[0]);
      return std::nullopt;
    }
    if (needs_value) {
      rule->apply(q, argv[i + 1]);
      i += 2;
    } else {
      q.cfg.verbose = false;  // -q
      i += 1;
    }
  }
  return q;
}

// "stdout"/"stderr" name the standard streams; no -o discards the factors.
std::string sink_path(const std::string &given) {
  if (given.empty()) return "/dev/null";
  if (given == "stdout") return "/dev/stdout";
  if (given == "stderr") return "/dev/stderr";
  return given;
}

// The tensor behind -f.  Text is parsed on the device; text the device
// parser refuses (a token the reference's stream would read only in part)
// and files that cannot be opened go through SymtensLoader, whose stream
// rules and messages then decide.  `clock_start` is moved past the host
// parse, which the reference does not time either.
SpSymtensor open_tensor(const std::string &path, Clock::time_point &clock_start) {
  if (SpSymtensor::is_spt(path)) return SpSymtensor::load_spt(path);
  if (std::ifstream(path).is_open()) {
    try {
      return SpSymtensor::load_tns(path);
    } catch (const std::runtime_error &) {
    }
  }
  SymtensLoader text(path);
  clock_start = Clock::now();
  return SpSymtensor(text.dim(), text.order(), text.unnz_inds(), text.unnzs());
}

struct Method {
  int code;
  const char *label;
  SymTuckerDecomp (SpSymtensor::*solve)(const Config &) const;
};

constexpr std::array<Method, 3> kMethods{{
    {0, "HOOI", &SpSymtensor::TuckerHOOI},
    {1, "HOQRI", &SpSymtensor::TuckerHOQRI},
    {2, "AltHOOI", &SpSymtensor::TuckerAltHOOI},
}};

void solve_and_write(const SpSymtensor &x, const Method &how, const Config &cfg, std::ostream &sink) {
  std::cout << "Running " << how.label << " algorithm" << std::endl;
  const auto start = Clock::now();
  SymTuckerDecomp result = (x.*how.solve)(cfg);
  std::cout << "---------- Time: " << elapsed_ms(start) << " ms ----------" << std::endl;
  FunctionTimer::printTimes();
  FunctionTimer::clear();
  result.print(sink);
}

}  // namespace

int main(int argc, char **argv) {
  const std::optional<Request> req = read_command_line(argc, argv);
  if (!req) return 1;
  try {
    auto start = Clock::now();
    const SpSymtensor x = open_tensor(req->tensor_path, start);
    std::cout << "Insertion time: " << elapsed_ms(start) << " ms" << std::endl;
    FunctionTimer::printTimes();
    FunctionTimer::clear();

    std::ofstream sink(sink_path(req->factor_sink));
    for (const Method &how : kMethods)
      if (req->which == -1 || req->which == how.code) solve_and_write(x, how, req->cfg, sink);
  } catch (const std::exception &e) {
    std::cerr << "symtucker: " << e.what() << std::endl;
    return 2;
  }
  return 0;
}
