// symtucker.hpp — the C++ entry points of SymProp, B200-native.
//
// The reference ships this header empty (include/symtucker.hpp, 0 bytes);
// its public API lives in include/detail/sparse/spsymtensor.hpp:26-65,
// include/detail/tucker.hpp:14-45, include/utils/loader.hpp:10-27 and
// include/utils/function_timer.hpp:9-36.  This header re-exports those names
// with the same signatures, implemented inline over the C ABI of
// include/symprop.h, so a program written against the reference compiles
// unchanged and runs its S3TTMc and Tucker loops on the GPU.
//
// Errors: the reference reports failures with assert / std::out_of_range /
// std::runtime_error; here every non-OK status of the C ABI is thrown as
// std::runtime_error carrying symprop_last_error() (std::out_of_range for
// an unsupported order, std::bad_alloc for out-of-memory).
#ifndef SYMPROP_SYMTUCKER_HPP
#define SYMPROP_SYMTUCKER_HPP

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <memory>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "symprop.h"

namespace symprop {

using real_t = double;     // include/utils/types.hpp:8
using order_t = uint32_t;  // types.hpp:9
using dim_t = uint32_t;    // types.hpp:10
using index_t = uint64_t;  // types.hpp:11

inline void check_status(int st) {
  if (st == SYMPROP_OK) return;
  std::string msg = std::string(symprop_status_string(st)) + ": " + symprop_last_error();
  if (st == SYMPROP_ERR_ORDER) throw std::out_of_range(msg);
  if (st == SYMPROP_ERR_OOM) throw std::bad_alloc();
  throw std::runtime_error(msg);
}

inline index_t symtens_size(index_t dim, index_t order) {
  return symprop_symtens_size((uint32_t)dim, (uint32_t)order);
}

inline std::vector<real_t> symtens_coeff(size_t dim, size_t N) {
  std::vector<real_t> c(symtens_size(dim, N));
  check_status(symprop_symtens_coeff((uint32_t)dim, (uint32_t)N, c.data()));
  return c;
}

// --------------------------------------------------------- FunctionTimer
// Accumulated phase table (include/utils/function_timer.hpp:9-36,
// src/utils/function_timer.cpp:12-80).  Phases of the GPU path are recorded
// with their device-measured durations.
class FunctionTimer {
 public:
  static void add(const std::string &name, double ms, long long calls = 1) {
    auto &t = table();
    t[name].first += ms;
    t[name].second += calls;
  }
  static void printTimes() {
    std::vector<std::pair<std::string, std::pair<double, long long>>> v(table().begin(),
                                                                        table().end());
    std::sort(v.begin(), v.end(),
              [](const auto &a, const auto &b) { return b.second.first < a.second.first; });
    std::cout << "Accumulated function times:\n";
    for (auto &e : v) {
      std::streamsize ss = std::cout.precision();
      std::cout << std::fixed << std::setprecision(3) << std::setw(10) << e.second.first
                << " ms  | " << std::setw(10) << e.second.second << " calls | " << e.first << "\n";
      std::cout.precision(ss);
      std::cout.unsetf(std::ios::fixed);
    }
  }
  static void clear() { table().clear(); }

 private:
  static std::map<std::string, std::pair<double, long long>> &table() {
    static std::map<std::string, std::pair<double, long long>> t;
    return t;
  }
};

// ----------------------------------------------------------------- Config
struct Config {  // include/detail/tucker.hpp:14-23
  dim_t rank = 2;
  index_t max_iter = 10;
  real_t rel_tol = 1e-6;
  real_t delta = 0.5;
  index_t seed = 0;
  std::string init = "rnd";
  // B200 additions (defaults give the reference's FP64 behaviour)
  int precision = SYMPROP_PREC_FP64;
  bool verbose = true;
  std::vector<real_t> init_factor;  // used when init == "user"

  Config() = default;
};

class SpSymtensor;

// --------------------------------------------------------- SymTuckerDecomp
class SymTuckerDecomp {  // include/detail/tucker.hpp:25-45
 public:
  real_t reconstruct_error(const SpSymtensor &target) const;
  void print(std::ostream &os) const {  // src/tucker.cpp:47-61
    os << "Mode-1 matricized C:\n";
    for (size_t i = 0; i < _rank; i++) {
      for (size_t j = 0; j < _core.size() / _rank; j++) os << _core[i * _rank + j] << ",";
      os << "\n";
    }
    os << "Factor U:\n";
    for (size_t i = 0; i < _dim; i++) {
      for (size_t j = 0; j < _rank; j++) os << _factor[i * _rank + j] << ",";
      os << "\n";
    }
  }
  const std::vector<real_t> &core() const { return _core; }
  const std::vector<real_t> &factor() const { return _factor; }
  index_t iterations() const { return _iters; }
  real_t error() const { return _error; }
  const std::vector<real_t> &error_trace() const { return _err_trace; }
  const std::vector<real_t> &relres_trace() const { return _res_trace; }
  double time_ms() const { return _time_ms; }

  friend class SpSymtensor;

 private:
  SymTuckerDecomp(const Config &c, dim_t dim, order_t order)
      : _dim(dim), _rank(c.rank), _order(order) {
    size_t cs = 1;
    for (order_t j = 0; j < order; j++) cs *= c.rank;
    _core.assign(cs, 0.0);
    _factor.assign((size_t)dim * c.rank, 0.0);
  }
  dim_t _dim;
  dim_t _rank;
  order_t _order;
  std::vector<real_t> _core;
  std::vector<real_t> _factor;
  std::vector<real_t> _err_trace, _res_trace;
  index_t _iters = 0;
  real_t _error = 0;
  real_t _core_norm = 0;
  double _time_ms = 0;
};

// --------------------------------------------------------------- matrix
// The reference's dense operations (include/detail/dense/matrixops.hpp:12-45,
// src/dense/matrixops.cpp:18-146) with the same signatures, computed on the
// GPU (symprop_gemmtn, ...).  As in the reference, a solver that does not
// converge prints its message and returns; the output then holds the last
// iterate.  Two differences: syevd and leftsvd leave A unchanged (LAPACK
// overwrites it with eigen- / singular vectors), and singular or
// eigenvector signs are the device solver's, not LAPACK's.
namespace matrix {

namespace detail {
struct Timed {  // records the call in FunctionTimer as START_FUNCTION_TIMER does
  const char *name;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  ~Timed() {
    FunctionTimer::add(
        name, std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
  }
};
inline void need(bool ok, const char *what) {
  if (!ok) throw std::runtime_error(std::string("matrix::") + what + ": operand has the wrong size");
}
inline void solved(int st, const char *message) {
  if (st == SYMPROP_ERR_NOCONV) std::printf("%s\n", message);
  else check_status(st);
}
}  // namespace detail

// U (nr x rank) = leading left singular vectors of A (nr x nc)
inline void leftsvd(std::vector<real_t> &A, std::vector<real_t> &U, size_t nr, size_t nc, size_t rank) {
  detail::Timed t{"leftsvd"};
  detail::need(A.size() >= nr * nc && U.size() >= nr * rank, "leftsvd");
  detail::solved(symprop_leftsvd(A.data(), U.data(), nr, nc, rank), "SVD failed to converge.");
}

// C (acol x bcol) = A^T B
inline void gemmtn(std::vector<real_t> &C, const std::vector<real_t> &A, const std::vector<real_t> &B,
                   size_t arow, size_t acol, size_t bcol) {
  detail::Timed t{"gemmtn"};
  detail::need(A.size() >= arow * acol && B.size() >= arow * bcol && C.size() >= acol * bcol, "gemmtn");
  check_status(symprop_gemmtn(C.data(), A.data(), B.data(), arow, acol, bcol));
}

// A (nr x nc) = Q of its QR decomposition
inline void qr(std::vector<real_t> &A, size_t nr, size_t nc) {
  detail::Timed t{"qr"};
  detail::need(A.size() >= nr * nc, "qr");
  check_status(symprop_qr(A.data(), nr, nc));
}

// U (dim x rank) = eigenvectors of the rank largest eigenvalues, ascending
inline void syevd(std::vector<real_t> &A, std::vector<real_t> &U, size_t dim, size_t rank) {
  detail::Timed t{"syevd"};
  detail::need(A.size() >= dim * dim && U.size() >= dim * rank, "syevd");
  detail::solved(symprop_syevd(A.data(), U.data(), dim, rank), "Eigendecomposition failed to converge.");
}

// C (I1 x I2) = A diag(row_coeff) B^T
inline void symgemm(std::vector<real_t> &C, const std::vector<real_t> &A, const std::vector<real_t> &B,
                    const std::vector<real_t> &row_coeff, size_t I1, size_t I2) {
  detail::Timed t{"symgemm"};
  const size_t m = row_coeff.size();
  detail::need(A.size() == I1 * m && B.size() == I2 * m && C.size() >= I1 * I2, "symgemm");
  check_status(symprop_symgemm(C.data(), A.data(), B.data(), row_coeff.data(), m, I1, I2));
}

// upper triangle of C (I1 x I1) = A diag(row_coeff) A^T
inline void symsyrk(std::vector<real_t> &C, const std::vector<real_t> &A, const std::vector<real_t> &row_coeff,
                    size_t I1) {
  detail::Timed t{"symsyrk"};
  const size_t m = row_coeff.size();
  detail::need(A.size() == I1 * m && C.size() == I1 * I1, "symsyrk");
  check_status(symprop_symsyrk(C.data(), A.data(), row_coeff.data(), m, I1));
}

}  // namespace matrix

// ------------------------------------------------------------ SpSymtensor
class SpSymtensor {  // include/detail/sparse/spsymtensor.hpp:24-65
 public:
  SpSymtensor(dim_t dim, order_t order, const std::vector<dim_t> &unnz_inds,
              const std::vector<real_t> &unnzs)
      : _dim(dim), _order(order), _unnz(unnzs.size()), _unnz_inds(unnz_inds), _unnzs(unnzs) {
    if (unnz_inds.size() != unnzs.size() * (size_t)order)
      throw std::runtime_error("unnz_inds size does not match order * nnz");
    symprop_tensor *t = nullptr;
    check_status(symprop_tensor_create(order, dim, unnz_inds.data(), unnzs.data(), unnzs.size(),
                                       &t));
    _t.reset(t);
    check_status(symprop_tensor_norm(t, &_norm));
    std::cout << "Finished creating compressed dtree\n";  // spsymtensor.cpp:26
  }

  // SymtensLoader + SpSymtensor in one step, with the .tns text parsed on
  // the device (symprop_tensor_load_tns); same tensor as
  // SpSymtensor(loader.dim(), loader.order(), loader.unnz_inds(), loader.unnzs())
  static SpSymtensor load_tns(const std::string &path) {
    symprop_tensor *t = nullptr;
    check_status(symprop_tensor_load_tns(path.c_str(), &t));
    return SpSymtensor(t);
  }
  // binary SPT1 tuple file (symprop_tensor_load_spt / save_spt)
  static SpSymtensor load_spt(const std::string &path) {
    symprop_tensor *t = nullptr;
    check_status(symprop_tensor_load_spt(path.c_str(), &t));
    return SpSymtensor(t);
  }
  void save_spt(const std::string &path) const { check_status(symprop_tensor_save_spt(_t.get(), path.c_str())); }
  // a file that starts with "SPT1" is binary, anything else .tns text
  static bool is_spt(const std::string &path) {
    std::ifstream f(path, std::ios::binary);
    char m[4] = {0, 0, 0, 0};
    return f.read(m, 4) && m[0] == 'S' && m[1] == 'P' && m[2] == 'T' && m[3] == '1';
  }
  static SpSymtensor load(const std::string &path) { return is_spt(path) ? load_spt(path) : load_tns(path); }

  order_t order() const { return _order; }
  dim_t dim() const { return _dim; }
  index_t size() const { return _unnz; }
  const std::vector<dim_t> &unnz_inds() const { return _unnz_inds; }
  const std::vector<real_t> &unnzs() const { return _unnzs; }
  real_t norm() const { return _norm; }

  // src/sparse/spsymtensor.cpp:30-110; res must hold dim * (packed ?
  // C(R+N-2,N-1) : R^(N-1)) values
  void S3TTMc(std::vector<real_t> &res, const std::vector<real_t> &U, dim_t R,
              bool partial_sym_res = false) const {
    size_t cols = partial_sym_res ? symtens_size(R, _order - 1)
                                  : (size_t)std::llround(std::pow((double)R, (double)_order - 1));
    if (res.size() != (size_t)_dim * cols) throw std::runtime_error("S3TTMc: res has wrong size");
    if (U.size() != (size_t)_dim * R) throw std::runtime_error("S3TTMc: U has wrong size");
    matrix::detail::Timed t{"S3TTMc"};
    check_status(
        symprop_s3ttmc(_t.get(), U.data(), R, partial_sym_res ? 1 : 0, res.data(), SYMPROP_FP64));
  }
  // FP32 variant (compensated FP32 accumulation)
  void S3TTMc(std::vector<float> &res, const std::vector<float> &U, dim_t R,
              bool partial_sym_res = false) const {
    check_status(
        symprop_s3ttmc(_t.get(), U.data(), R, partial_sym_res ? 1 : 0, res.data(), SYMPROP_FP32));
  }

  SymTuckerDecomp TuckerHOOI(const Config &c) const { return run(c, SYMPROP_HOOI); }
  SymTuckerDecomp TuckerHOQRI(const Config &c) const { return run(c, SYMPROP_HOQRI); }
  SymTuckerDecomp TuckerAltHOOI(const Config &c) const { return run(c, SYMPROP_ALTHOOI); }

  const symprop_tensor *handle() const { return _t.get(); }

 private:
  struct Del {
    void operator()(symprop_tensor *t) const { symprop_tensor_destroy(t); }
  };

  explicit SpSymtensor(symprop_tensor *t) : _t(t) {
    uint64_t nnz = 0;
    check_status(symprop_tensor_order(t, &_order));
    check_status(symprop_tensor_dim(t, &_dim));
    check_status(symprop_tensor_nnz(t, &nnz));
    _unnz = (index_t)nnz;
    _unnz_inds.resize((size_t)nnz * _order);
    _unnzs.resize((size_t)nnz);
    check_status(symprop_tensor_copy_nonzeros(t, _unnz_inds.data(), _unnzs.data()));
    check_status(symprop_tensor_norm(t, &_norm));
    std::cout << "Finished creating compressed dtree\n";  // spsymtensor.cpp:26
  }

  SymTuckerDecomp run(const Config &c, int alg) const {
    SymTuckerDecomp d(c, _dim, _order);
    symprop_config cfg{};
    cfg.rank = c.rank;
    cfg.max_iter = c.max_iter;
    cfg.rel_tol = c.rel_tol;
    cfg.delta = c.delta;
    cfg.seed = c.seed;
    cfg.precision = c.precision;
    cfg.verbose = c.verbose ? 1 : 0;
    if (c.init == "rnd") cfg.init = SYMPROP_INIT_RND;
    else if (c.init == "hoevd") cfg.init = SYMPROP_INIT_HOEVD;
    else if (c.init == "hosvd") cfg.init = SYMPROP_INIT_HOSVD;
    else if (c.init == "user") cfg.init = SYMPROP_INIT_USER;
    else cfg.init = SYMPROP_INIT_RND;  // unknown names leave the random init (spsymtensor.cpp:339-383)
    symprop_result r{};
    r.core = d._core.data();
    r.factor = d._factor.data();
    d._err_trace.assign(c.max_iter, 0.0);
    d._res_trace.assign(c.max_iter, 0.0);
    r.error_trace = d._err_trace.data();
    r.relres_trace = d._res_trace.data();
    r.trace_cap = c.max_iter;
    if (cfg.init == SYMPROP_INIT_USER) {
      if (c.init_factor.size() != (size_t)_dim * c.rank)
        throw std::runtime_error("init_factor must hold dim * rank values");
      r.init_factor = c.init_factor.data();
    }
    check_status(symprop_tucker(_t.get(), &cfg, alg, &r));
    d._iters = r.iterations;
    d._err_trace.resize(r.iterations);
    d._res_trace.resize(r.iterations);
    d._error = r.error;
    d._core_norm = r.core_norm;
    d._time_ms = r.time_ms;
    static const char *names[] = {"TuckerHOOI", "TuckerHOQRI", "TuckerAltHOOI"};
    FunctionTimer::add(names[alg], r.time_ms);
    FunctionTimer::add("S3TTMc", r.s3ttmc_ms, (long long)r.iterations);
    FunctionTimer::add("dense steps", r.dense_ms, (long long)r.iterations);
    return d;
  }

  dim_t _dim;
  order_t _order;
  index_t _unnz;
  real_t _norm = 0;
  std::unique_ptr<symprop_tensor, Del> _t;
  std::vector<dim_t> _unnz_inds;
  std::vector<real_t> _unnzs;
};

// ||X||, ||C|| based error (src/tucker.cpp:40-45)
inline real_t SymTuckerDecomp::reconstruct_error(const SpSymtensor &target) const {
  real_t sp = target.norm();
  real_t cn = 0;
  for (real_t v : _core) cn += v * v;
  cn = std::sqrt(cn);
  return std::sqrt(sp * sp - cn * cn) / sp;
}

// ------------------------------------------------------------ SymtensLoader
class SymtensLoader {  // include/utils/loader.hpp:10-27, src/utils/loader.cpp:8-36
 public:
  explicit SymtensLoader(const std::string &filename) : _filename(filename) {
    std::ifstream file(filename);
    if (!file.is_open()) {
      std::cerr << "Error opening file: " << filename << std::endl;
      throw std::runtime_error("Error opening file in SymtensLoader");
    }
    file >> _order >> _dim;
    std::vector<dim_t> idx;
    while (true) {
      idx.clear();
      for (order_t i = 0; i < _order; i++) {
        dim_t v;
        file >> v;
        idx.push_back(v);
      }
      real_t val;
      file >> val;
      if (!file.good()) break;
      std::sort(idx.begin(), idx.end());
      _unnzs.push_back(val);
      _unnz_inds.insert(_unnz_inds.end(), idx.begin(), idx.end());
    }
  }
  const std::vector<dim_t> &unnz_inds() const { return _unnz_inds; }
  const std::vector<real_t> &unnzs() const { return _unnzs; }
  order_t order() const { return _order; }
  dim_t dim() const { return _dim; }

 private:
  std::string _filename;
  std::vector<dim_t> _unnz_inds;
  std::vector<real_t> _unnzs;
  order_t _order = 0;
  dim_t _dim = 0;
};

}  // namespace symprop

#endif  // SYMPROP_SYMTUCKER_HPP
