/*
 * skema.hpp -- the C++ drop-in layer over the C ABI (skema_c.h).
 *
 * It keeps the names and call pattern of the reference's sketch API, so a
 * driver written against Skema's headers swaps it in:
 *   - the global typedefs scalar_type, ordinal_type, size_type, range_type,
 *     matrix_type, vector_type, crs_matrix_type (src/Skema_Utils.hpp:9-33),
 *     here host containers (column-major, LayoutLeft) instead of Kokkos views;
 *   - the enum structs Skema::Solver_Method, Kernel_Map, DimRedux_Map, ...
 *     (src/Skema_Utils.hpp:38-80);
 *   - Skema::AlgParams with its fields, defaults, parse() and print()
 *     (src/Skema_AlgParams.hpp:12-90, src/Skema_AlgParams.cpp:10-606) and the
 *     parse_* helpers, build_arg_list and check_and_print_unused_args;
 *   - Skema::GaussDimRedux / SparseSignDimRedux with lmap / rmap
 *     (src/Skema_DimRedux.hpp:60-268);
 *   - Skema::SketchySVD<MatrixType, DimReduxT> and SketchySPD: ctor(AlgParams),
 *     linear_update, low_rank_approx, compute_residuals, save_history
 *     (src/Skema_SketchySVD.hpp:11-108);
 *   - Skema::sketchysvd(matrix, algParams) (src/Skema_SketchySVD.cpp:1244,1408)
 *     and Skema::read_matrix<T>(path) (src/Skema_IO.hpp:13-21).
 * Everything computes in the CUDA library: matrices are FP64 on the host, as
 * the reference holds them, and are handed to the library in FP32 (its input
 * type); the fixed-rank approximation comes back in FP64. Failed calls throw
 * std::runtime_error with the library's message, so the reference's
 * try / catch -> exit(EXIT_FAILURE) pattern (src/Skema_SketchySVD.cpp:1280-1307)
 * behaves the same. Link with libskema_b200.so. C++17.
 */
#ifndef SKEMA_HPP
#define SKEMA_HPP

#include <algorithm>
#include <charconv>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

#include "skema_c.h"

namespace Skema {
namespace host {

// Dense column-major FP64 matrix (the reference's Kokkos::View<double**, LayoutLeft>).
class Matrix {
 public:
  Matrix() = default;
  Matrix(const std::string& label, std::size_t m, std::size_t n) : label_(label), m_(m), n_(n), v_(m * n, 0.0) {}
  Matrix(std::size_t m, std::size_t n) : Matrix("", m, n) {}
  std::size_t extent(int r) const { return r == 0 ? m_ : n_; }
  double& operator()(std::size_t i, std::size_t j) { return v_[i + j * m_]; }
  const double& operator()(std::size_t i, std::size_t j) const { return v_[i + j * m_]; }
  double* data() { return v_.data(); }
  const double* data() const { return v_.data(); }
  const std::string& label() const { return label_; }

 private:
  std::string label_;
  std::size_t m_ = 0, n_ = 0;
  std::vector<double> v_;
};

// FP64 vector (Kokkos::View<double*, LayoutLeft>).
class Vector {
 public:
  Vector() = default;
  Vector(const std::string& label, std::size_t n) : label_(label), v_(n, 0.0) {}
  explicit Vector(std::size_t n) : Vector("", n) {}
  std::size_t extent(int) const { return v_.size(); }
  double& operator()(std::size_t i) { return v_[i]; }
  const double& operator()(std::size_t i) const { return v_[i]; }
  double* data() { return v_.data(); }
  const double* data() const { return v_.data(); }

 private:
  std::string label_;
  std::vector<double> v_;
};

// CRS FP64 matrix (KokkosSparse::CrsMatrix<double, int, device, void, size_t>):
// row_map (numRows + 1 offsets), entries (column indices), values.
class Crs {
 public:
  Crs() = default;
  Crs(const std::string& label, std::size_t nrows, std::size_t ncols, std::size_t nnz, std::vector<double> values,
      std::vector<std::size_t> row_map, std::vector<int> entries)
      : row_map(std::move(row_map)), entries(std::move(entries)), values(std::move(values)), label_(label),
        nrows_(nrows), ncols_(ncols) {
    if (this->row_map.size() != nrows + 1 || this->entries.size() != nnz || this->values.size() != nnz)
      throw std::runtime_error("crs_matrix_type: array sizes do not match nrows / nnz");
  }
  std::size_t numRows() const { return nrows_; }
  std::size_t numCols() const { return ncols_; }
  std::size_t nnz() const { return values.size(); }
  std::vector<std::size_t> row_map;
  std::vector<int> entries;
  std::vector<double> values;

 private:
  std::string label_;
  std::size_t nrows_ = 0, ncols_ = 0;
};

}  // namespace host
}  // namespace Skema

// The reference's global typedefs (src/Skema_Utils.hpp:9-33).
using scalar_type = double;
using ordinal_type = int;
using size_type = std::size_t;
using range_type = std::pair<size_type, size_type>;
using matrix_type = Skema::host::Matrix;
using vector_type = Skema::host::Vector;
using crs_matrix_type = Skema::host::Crs;

namespace Skema {

// ---- enums (src/Skema_Utils.hpp:38-80), same members, order and names ----
struct Matrix_Type {
  enum type { DENSE, SPARSE };
  static constexpr unsigned num_types = 2;
  static constexpr type types[] = {DENSE, SPARSE};
  static constexpr const char* names[] = {"dense", "sparse"};
};
struct Solver_Method {
  enum type { ISVD, SKETCH, PRIMME };
  static constexpr unsigned num_types = 3;
  static constexpr type types[] = {ISVD, SKETCH, PRIMME};
  static constexpr const char* names[] = {"isvd", "sketch", "primme"};
};
struct Decomposition_Type {
  enum type { EIG, EIGS, SVD, SVDS };
  static constexpr unsigned num_types = 4;
  static constexpr type types[] = {EIG, EIGS, SVD, SVDS};
  static constexpr const char* names[] = {"eig", "eigs", "svd", "svds"};
};
struct Kernel_Map {
  enum type { NONE, GAUSSRBF };
  static constexpr unsigned num_types = 2;
  static constexpr type types[] = {NONE, GAUSSRBF};
  static constexpr const char* names[] = {"none", "gaussrbf"};
};
struct Sampler_Type {
  enum type { RESERVOIR };
  static constexpr unsigned num_types = 1;
  static constexpr type types[] = {RESERVOIR};
  static constexpr const char* names[] = {"reservoir"};
};
struct DimRedux_Map {
  enum type { GAUSS, SPARSE_SIGN };
  static constexpr unsigned num_types = 2;
  static constexpr type types[] = {GAUSS, SPARSE_SIGN};
  static constexpr const char* names[] = {"gauss", "sparse-sign"};
};
// Arithmetic of the sketch contractions (new; SKEMA_PREC_*).
struct Precision {
  enum type { FP32, BF16, FP8 };
  static constexpr unsigned num_types = 3;
  static constexpr type types[] = {FP32, BF16, FP8};
  static constexpr const char* names[] = {"fp32", "bf16", "fp8"};
};
// SketchySPD approximation (new; SKEMA_SPD_*).
struct Spd_Approx {
  enum type { NYSTROM, REFERENCE_STEPS };
  static constexpr unsigned num_types = 2;
  static constexpr type types[] = {NYSTROM, REFERENCE_STEPS};
  static constexpr const char* names[] = {"nystrom", "reference-steps"};
};

// ---- argument parsing (src/Skema_AlgParams.cpp:242-606) ------------------
// Skema::error (src/Skema_AlgParams.cpp:59-62): report and throw.
[[noreturn]] inline void error(std::string s) {
  std::cerr << "FATAL ERROR: " << s << std::endl;
  throw std::runtime_error(s);
}

namespace detail {
// Position of a flag in args: "--name" or the bare "name".
inline std::ptrdiff_t find_flag(const std::vector<std::string>& args, const std::string& flag) {
  for (std::size_t i = 0; i < args.size(); ++i)
    if (args[i] == flag) return (std::ptrdiff_t)i;
  if (flag.size() > 2 && flag.compare(0, 2, "--") == 0) {
    const std::string bare = flag.substr(2);
    for (std::size_t i = 0; i < args.size(); ++i)
      if (args[i] == bare) return (std::ptrdiff_t)i;
  }
  return -1;
}
inline void erase(std::vector<std::string>& args, std::ptrdiff_t i, std::ptrdiff_t n) {
  args.erase(args.begin() + i, args.begin() + std::min<std::ptrdiff_t>(i + n, (std::ptrdiff_t)args.size()));
}
template <typename T>
std::string range_msg(const std::string& flag, const std::string& v, T lo, T hi) {
  return "Bad input: " + flag + " " + v + ",  must be in the range (" + std::to_string(lo) + ", " +
         std::to_string(hi) + ")";
}
}  // namespace detail

inline std::vector<std::string> build_arg_list(int argc, char** argv) {
  std::vector<std::string> a;
  for (int i = 1; i < argc; ++i) a.emplace_back(argv[i]);
  return a;
}

inline bool parse_bool(std::vector<std::string>& args, const std::string& cl_arg_on, const std::string& cl_arg_off,
                       bool default_value) {
  std::ptrdiff_t i = detail::find_flag(args, cl_arg_on);
  if (i >= 0) {
    detail::erase(args, i, 1);
    return true;
  }
  i = detail::find_flag(args, cl_arg_off);
  if (i >= 0) {
    detail::erase(args, i, 1);
    return false;
  }
  return default_value;
}

inline int parse_int(std::vector<std::string>& args, const std::string& cl_arg, int default_value, int min = 0,
                     int max = 100) {
  int val = default_value;
  const std::ptrdiff_t i = detail::find_flag(args, cl_arg);
  if (i >= 0) {
    if (i + 1 >= (std::ptrdiff_t)args.size()) {
      detail::erase(args, i, 1);
      return val;
    }
    const std::string& s = args[i + 1];
    if (s == "inf" || s == "Inf") {
      val = INT_MAX;
    } else {
      char* end = nullptr;
      const long v = std::strtol(s.c_str(), &end, 10);
      if (end == s.c_str()) error("Unparseable input: " + cl_arg + " " + s + ", must be an integer");
      val = (int)v;
    }
    detail::erase(args, i, 2);
  }
  if (val < min || val > max) error(detail::range_msg(cl_arg, std::to_string(val), min, max));
  return val;
}

inline double parse_real(std::vector<std::string>& args, const std::string& cl_arg, double default_value,
                         double min = 0.0, double max = 1.0) {
  double val = default_value;
  const std::ptrdiff_t i = detail::find_flag(args, cl_arg);
  if (i >= 0) {
    if (i + 1 >= (std::ptrdiff_t)args.size()) {
      detail::erase(args, i, 1);
      return val;
    }
    const std::string& s = args[i + 1];
    char* end = nullptr;
    val = std::strtod(s.c_str(), &end);
    if (end == s.c_str()) error("Unparseable input: " + cl_arg + " " + s + ", must be a double");
    detail::erase(args, i, 2);
  }
  if (val < min || val > max) error(detail::range_msg(cl_arg, std::to_string(val), min, max));
  return val;
}

inline std::string parse_string(std::vector<std::string>& args, const std::string& cl_arg,
                                const std::string& default_value) {
  const std::ptrdiff_t i = detail::find_flag(args, cl_arg);
  if (i < 0) return default_value;
  if (i + 1 >= (std::ptrdiff_t)args.size()) {
    detail::erase(args, i, 1);
    return default_value;
  }
  std::string v = args[i + 1];
  detail::erase(args, i, 2);
  return v;
}

inline std::filesystem::path parse_filepath(std::vector<std::string>& args, const std::string& cl_arg,
                                            const std::string& default_value) {
  return std::filesystem::path(parse_string(args, cl_arg, default_value));
}

// Index of the value in names, or default_value when the flag is absent.
inline unsigned parse_enum_index(std::vector<std::string>& args, const std::string& cl_arg, unsigned default_value,
                                 unsigned num_values, const char* const* names) {
  const std::ptrdiff_t i = detail::find_flag(args, cl_arg);
  if (i < 0) return default_value;
  if (i + 1 >= (std::ptrdiff_t)args.size()) {
    detail::erase(args, i, 1);
    return default_value;
  }
  const std::string v = args[i + 1];
  detail::erase(args, i, 2);
  for (unsigned k = 0; k < num_values; ++k)
    if (v == names[k]) return k;
  std::string all;
  for (unsigned k = 0; k < num_values; ++k) all += std::string(k ? ", " : "") + names[k];
  error("Bad input: " + cl_arg + " " + v + ",  must be one of the values: " + all + ".");
}

inline std::vector<int> parse_int_array(std::vector<std::string>& args, const std::string& cl_arg,
                                        const std::vector<int>& default_value, int min = 1, int max = INT_MAX) {
  const std::ptrdiff_t i = detail::find_flag(args, cl_arg);
  if (i < 0) return default_value;
  if (i + 1 >= (std::ptrdiff_t)args.size()) {
    detail::erase(args, i, 1);
    return default_value;
  }
  const std::string s = args[i + 1];
  const std::string shape = ", must be of the form [int,...,int] with no spaces";
  if (s.empty() || s[0] != '[') error("Unparseable input: " + cl_arg + " " + s + shape);
  std::string body = s.substr(1);
  if (!body.empty() && body.back() == ']') body.pop_back();
  std::vector<int> vals;
  std::size_t at = 0;
  while (at <= body.size()) {
    const std::size_t comma = std::min(body.find(',', at), body.size());
    const std::string tok = body.substr(at, comma - at);
    if (!tok.empty()) {
      char* end = nullptr;
      const long v = std::strtol(tok.c_str(), &end, 10);
      if (end == tok.c_str() || *end != '\0') error("Unparseable input: " + cl_arg + " " + tok + shape);
      if (v < min || v > max) error(detail::range_msg(cl_arg, tok, min, max));
      vals.push_back((int)v);
    }
    at = comma + 1;
  }
  detail::erase(args, i, 2);
  return vals;
}

inline bool check_and_print_unused_args(const std::vector<std::string>& args, std::ostream& out) {
  if (args.empty()) return false;
  out << "Error!  Unknown command line arguments: ";
  for (const std::string& a : args) out << a << " ";
  out << std::endl << std::endl;
  return true;
}

// ---- AlgParams (src/Skema_AlgParams.hpp:12-90) ---------------------------
struct AlgParams {
  Solver_Method::type solver = Solver_Method::ISVD;
  Decomposition_Type::type decomposition_type = Decomposition_Type::SVDS;
  std::filesystem::path inputfilename, outputfilename, history_filename, debug_filename;
  bool issparse = false;
  bool issymmetric = false;
  size_t matrix_m = 0, matrix_n = 0, matrix_nnz = 0;
  size_t rank = 1;
  int num_passes = 1;
  int print_level = 0;
  bool debug = false;
  size_t window = 1;
  bool hist = false;
  bool rayleigh_ritz_pass = false;
  double normalize_matrix = 0.0;
  // ISVD / PRIMME / sampling options: carried so a driver compiles; this
  // library implements the sketch path only.
  bool isvd_dense_solver = false, isvd_initial_guess = false, isvd_compute_residual_iters = false;
  size_t isvd_rank_add_factor = 0;
  std::filesystem::path primme_outputFile;
  double primme_eps = 1e-10;
  int primme_initSize = 0, primme_maxBasisSize = 0, primme_minRestartSize = 0, primme_maxBlockSize = 0,
      primme_printLevel = 0, primme_maxMatvecs = 0, primme_maxIter = 0;
  bool primme_locking = true;
  std::string primme_method, primme_methodStage2;
  double isvd_convtest_eps = 1e-1;
  int isvd_convtest_skip = 0;
  Sampler_Type::type isvd_sampler = Sampler_Type::RESERVOIR;
  bool isvd_sampling = false;
  size_t isvd_num_samples = 0;
  // sketch options
  size_t sketch_range = 1, sketch_core = 1;
  double sketch_eta = 1.0, sketch_nu = 1.0;
  std::vector<int> seeds{0, 1, 2, 3};
  bool force_three_sketch = false;
  bool sketch_compute_svals_iters = false;
  DimRedux_Map::type dim_redux = DimRedux_Map::GAUSS;
  Kernel_Map::type kernel_func = Kernel_Map::NONE;
  double kernel_gamma = 1.0;
  // new: arithmetic of the contractions, CUDA device, SketchySPD approximation
  Precision::type precision = Precision::FP32;
  int device = 0;
  Spd_Approx::type spd_approx = Spd_Approx::NYSTROM;

  AlgParams() = default;

  // The sketch flags, consumed from args (src/Skema_AlgParams.cpp:242-330).
  void parse(std::vector<std::string>& args) {
    inputfilename = parse_filepath(args, "--input", inputfilename.string());
    debug_filename = parse_filepath(args, "--debug-file", debug_filename.string());
    history_filename = parse_filepath(args, "--history-file", history_filename.string());
    issparse = parse_bool(args, "--sparse", "--dense", issparse);
    issymmetric = parse_bool(args, "--symmetric", "--asymmetric", issymmetric);
    matrix_m = (size_t)parse_int(args, "--m", (int)matrix_m, 0, INT_MAX);
    matrix_n = (size_t)parse_int(args, "--n", (int)matrix_n, 0, INT_MAX);
    rank = (size_t)parse_int(args, "--rank", (int)rank, 1, INT_MAX);
    num_passes = parse_int(args, "--num-passes", num_passes, 1, INT_MAX);
    solver = Solver_Method::types[parse_enum_index(args, "--solver", solver, Solver_Method::num_types,
                                                   Solver_Method::names)];
    print_level = parse_int(args, "--print-level", print_level, 0, 5);
    debug = parse_bool(args, "--debug", "--debug-off", debug);
    window = (size_t)parse_int(args, "--window", (int)window, 1, INT_MAX);
    dim_redux = DimRedux_Map::types[parse_enum_index(args, "--model", dim_redux, DimRedux_Map::num_types,
                                                     DimRedux_Map::names)];
    sketch_range = (size_t)parse_int(args, "--range", (int)sketch_range, 0, INT_MAX);
    sketch_core = (size_t)parse_int(args, "--core", (int)sketch_core, 0, INT_MAX);
    seeds = parse_int_array(args, "--seeds", seeds, 0, INT_MAX);
    sketch_eta = parse_real(args, "--eta", sketch_eta, 0.0, INFINITY);
    sketch_nu = parse_real(args, "--nu", sketch_nu, 0.0, INFINITY);
    force_three_sketch = parse_bool(args, "--force-three-sketch", "--force-three-sketch-off", force_three_sketch);
    sketch_compute_svals_iters = parse_bool(args, "--sketch-compute-svals-iters",
                                            "--sketch-compute-svals-iters-off", sketch_compute_svals_iters);
    kernel_func = Kernel_Map::types[parse_enum_index(args, "--kernel", kernel_func, Kernel_Map::num_types,
                                                     Kernel_Map::names)];
    kernel_gamma = parse_real(args, "--gamma", kernel_gamma, 0.0, INFINITY);
    normalize_matrix = parse_real(args, "--normalize-matrix", normalize_matrix, 0.0, INFINITY);
    precision = Precision::types[parse_enum_index(args, "--precision", precision, Precision::num_types,
                                                  Precision::names)];
    spd_approx = Spd_Approx::types[parse_enum_index(args, "--spd-approx", spd_approx, Spd_Approx::num_types,
                                                    Spd_Approx::names)];
    device = parse_int(args, "--device", device, 0, INT_MAX);
  }

  void print(std::ostream& out) const {
    out << "  solver = " << Solver_Method::names[solver] << "\n  window = " << window << "\n  rank = " << rank
        << "\n  sketch_range = " << sketch_range << "\n  sketch_core = " << sketch_core
        << "\n  sketch_eta = " << sketch_eta << "\n  sketch_nu = " << sketch_nu
        << "\n  model = " << DimRedux_Map::names[dim_redux] << "\n  kernel = " << Kernel_Map::names[kernel_func]
        << "\n  gamma = " << kernel_gamma << "\n  precision = " << Precision::names[precision] << "\n  seeds = [";
    for (std::size_t i = 0; i < seeds.size(); ++i) out << (i ? "," : "") << seeds[i];
    out << "]" << std::endl;
  }

  static void print_help(std::ostream& out) {
    out << "Sketch options:\n"
        << "  --solver isvd|sketch|primme\n  --model gauss|sparse-sign\n  --range <int>\n  --core <int>\n"
        << "  --eta <real>\n  --nu <real>\n  --seeds [int,...,int]\n  --force-three-sketch\n"
        << "  --sketch-compute-svals-iters\n  --kernel none|gaussrbf\n  --gamma <real>\n"
        << "  --precision fp32|bf16|fp8\n  --spd-approx nystrom|reference-steps\n  --device <int>" << std::endl;
  }

  // The C ABI's parameter block for a context over A (three-sketch unless spd).
  skema_params to_c(int32_t kind, bool spd) const {
    skema_params p;
    skema_params_init(&p);
    p.matrix_m = (int64_t)matrix_m;
    p.matrix_n = (int64_t)matrix_n;
    p.rank = (int64_t)rank;
    p.sketch_range = (int64_t)sketch_range;
    p.sketch_core = (int64_t)sketch_core;
    p.window = (int64_t)window;
    p.sketch_eta = sketch_eta;
    p.sketch_nu = sketch_nu;
    for (int i = 0; i < 4; ++i) p.seeds[i] = i < (int)seeds.size() ? seeds[i] : i;
    p.dim_redux = kind;
    p.issparse = issparse ? 1 : 0;
    p.issymmetric = spd ? 1 : 0;
    p.force_three_sketch = spd ? 0 : 1;
    p.kernel_func = kernel_func == Kernel_Map::GAUSSRBF ? SKEMA_KERNEL_GAUSSRBF : SKEMA_KERNEL_NONE;
    p.kernel_gamma = kernel_gamma;
    p.precision = (int32_t)precision;
    p.device = device;
    p.spd_approx = (int32_t)spd_approx;
    return p;
  }
};

// ---- library calls ---------------------------------------------------------
namespace detail {
inline void check(int st, const char* msg) {
  if (st != SKEMA_OK) throw std::runtime_error(std::string("skema: ") + (msg ? msg : "") + " (status " +
                                               std::to_string(st) + ")");
}
inline void check_ctx(int st, const skema_ctx* c) {
  if (st != SKEMA_OK) check(st, skema_last_error(c));
}
// A dense FP64 host matrix as FP32 column-major (the library's input type).
inline std::vector<float> to_f32(const matrix_type& A) {
  const std::size_t n = A.extent(0) * A.extent(1);
  std::vector<float> f(n);
  for (std::size_t i = 0; i < n; ++i) f[i] = (float)A.data()[i];
  return f;
}
struct CsrF32 {
  std::vector<int64_t> rowptr;
  std::vector<int32_t> col;
  std::vector<float> val;
};
inline CsrF32 to_f32(const crs_matrix_type& A) {
  CsrF32 o;
  o.rowptr.assign(A.row_map.begin(), A.row_map.end());
  o.col.assign(A.entries.begin(), A.entries.end());
  o.val.resize(A.values.size());
  for (std::size_t i = 0; i < A.values.size(); ++i) o.val[i] = (float)A.values[i];
  return o;
}
inline matrix_type from_f32(const std::vector<float>& f, std::size_t m, std::size_t n, const std::string& label) {
  matrix_type C(label, m, n);
  for (std::size_t i = 0; i < m * n; ++i) C.data()[i] = (double)f[i];
  return C;
}
// Shortest decimal that reads back to the same double (as the JSON writer
// of the reference's save_history prints numbers).
inline std::string num(double x) {
  if (!std::isfinite(x)) return "null";
  char b[64];
  const auto r = std::to_chars(b, b + sizeof b, x);
  std::string s(b, r.ptr);
  if (s.find_first_of(".e") == std::string::npos) s += ".0";
  return s;
}
}  // namespace detail

// Skema::read_matrix (src/Skema_IO.hpp:13-21): .mtx array -> matrix_type,
// .mtx coordinate or .bin -> crs_matrix_type.
template <typename T>
T read_matrix(const std::filesystem::path& path);

template <>
inline matrix_type read_matrix<matrix_type>(const std::filesystem::path& path) {
  skema_dense d{};
  detail::check(skema_read_dense(path.string().c_str(), &d), skema_last_error(nullptr));
  matrix_type A(path.stem().string(), (std::size_t)d.nrow, (std::size_t)d.ncol);
  std::copy(d.data, d.data + d.nrow * d.ncol, A.data());
  skema_dense_free(&d);
  return A;
}

template <>
inline crs_matrix_type read_matrix<crs_matrix_type>(const std::filesystem::path& path) {
  skema_crs a{};
  detail::check(skema_read_crs(path.string().c_str(), &a), skema_last_error(nullptr));
  std::vector<std::size_t> rm(a.rowptr, a.rowptr + a.nrow + 1);
  std::vector<int> ent(a.col, a.col + a.nnz);
  std::vector<double> val(a.val, a.val + a.nnz);
  crs_matrix_type A(path.stem().string(), (std::size_t)a.nrow, (std::size_t)a.ncol, (std::size_t)a.nnz,
                    std::move(val), std::move(rm), std::move(ent));
  skema_crs_free(&a);
  return A;
}

// ---- --debug-file dumps ----------------------------------------------------
namespace detail {
inline FILE* open_dump(const std::string& fname) {
  FILE* f = std::fopen(fname.c_str(), "w");
  if (!f) throw std::runtime_error("skema: cannot write " + fname);
  return f;
}
// Impl::write (src/Skema_Common.hpp:164-184): a matrix as one line per row of
// "%.16f " entries, a vector as one "%.16f" value per line.
inline void write_text(const std::string& fname, const matrix_type& A) {
  FILE* f = open_dump(fname);
  for (size_type i = 0; i < A.extent(0); ++i) {
    for (size_type j = 0; j < A.extent(1); ++j) std::fprintf(f, "%.16f ", A(i, j));
    std::fprintf(f, "\n");
  }
  std::fclose(f);
}
inline void write_text(const std::string& fname, const vector_type& v) {
  FILE* f = open_dump(fname);
  for (size_type i = 0; i < v.extent(0); ++i) std::fprintf(f, "%.16f\n", v(i));
  std::fclose(f);
}
// A map as the reference's constructors dump it (src/Skema_DimRedux.hpp:
// 124-127, 264-267): Gauss values (nr x nc, column-major) to <stem>_<label>.txt
// as write_text lines; SparseSign (z entries per stored row, row-major) to
// <stem>_<label>.mtx as a MatrixMarket coordinate file with 1-based indices,
// a row's entries in stored order (repeated columns kept).
inline void write_map_dump(const std::string& stem, const std::string& label, int64_t nr, int64_t nc, int z,
                           const std::vector<double>& vals, const std::vector<int32_t>& idx) {
  if (z == 0) {
    FILE* f = open_dump(stem + "_" + label + ".txt");
    for (int64_t i = 0; i < nr; ++i) {
      for (int64_t j = 0; j < nc; ++j) std::fprintf(f, "%.16f ", vals[(size_t)(i + j * nr)]);
      std::fprintf(f, "\n");
    }
    std::fclose(f);
    return;
  }
  FILE* f = open_dump(stem + "_" + label + ".mtx");
  std::fprintf(f, "%%%%MatrixMarket matrix coordinate real general\n");
  std::fprintf(f, "%lld %lld %lld\n", (long long)nr, (long long)nc, (long long)nr * z);
  for (int64_t i = 0; i < nr; ++i)
    for (int t = 0; t < z; ++t)
      std::fprintf(f, "%lld %d %.17g\n", (long long)(i + 1), idx[(size_t)(i * z + t)] + 1, vals[(size_t)(i * z + t)]);
  std::fclose(f);
}
// The file stem of --debug-file (debug_filename.filename().stem()); the
// dumps go to the working directory, as the reference writes them.
inline std::string debug_stem(const std::filesystem::path& debug_filename) {
  return debug_filename.empty() ? std::string() : debug_filename.filename().stem().string();
}
}  // namespace detail

// ---- DimRedux (src/Skema_DimRedux.hpp:60-268) -----------------------------
struct DimReduxStats {
  scalar_type initialize{0.0};
  scalar_type map{0.0};
};

template <typename Derived, int32_t KIND>
class DimRedux {
 public:
  static constexpr int32_t kind = KIND;
  DimRedux(const size_type nrow_, const size_type ncol_, const ordinal_type seed_, const std::string label_,
           const bool debug_ = false, const std::filesystem::path debug_filename_ = "",
           const bool init_transposed_ = false, int device = 0)
      : nrow(nrow_), ncol(ncol_), seed(seed_), label(label_), debug(debug_), debug_filename(debug_filename_),
        init_transposed(init_transposed_) {
    const auto t0 = std::chrono::steady_clock::now();
    skema_dimredux* h = nullptr;
    const int st = skema_dimredux_create(KIND, (int64_t)nrow, (int64_t)ncol, seed, device, &h);
    if (st != SKEMA_OK) detail::check(st, "skema_dimredux_create failed");
    map_ = std::shared_ptr<skema_dimredux>(h, Free{});
    stats.initialize = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (!debug_filename.empty()) {
      std::vector<double> v;
      std::vector<int32_t> ix;
      export_map(v, ix);
      const int z = KIND == SKEMA_MAP_SPARSE_SIGN ? (int)(v.size() / std::max<size_type>(nrow, 1)) : 0;
      detail::write_map_dump(detail::debug_stem(debug_filename), label, (int64_t)nrow, (int64_t)ncol, z, v, ix);
    }
  }

  // lmap: for a dense B, op(M(:, idx)) op(B), where op(M) is transposed when
  // exactly one of transA == 'T' and init_transposed holds
  // (src/Skema_DimRedux_Gauss.cpp:10-33, src/Skema_DimRedux_SparseSign.cpp:9-31).
  matrix_type lmap(const scalar_type* alpha, const matrix_type& B, const scalar_type* beta, char transA = 'N',
                   char transB = 'N', const range_type idx = range_type(0, 0)) {
    if (init_transposed) transA = (transA == 'N') ? 'T' : 'N';
    return dense_product(true, *alpha, B, *beta, transA, transB, idx);
  }
  // rmap: for a dense A, op(A) op(M) (src/Skema_DimRedux_Gauss.cpp:35-52,
  // src/Skema_DimRedux_SparseSign.cpp:33-51).
  matrix_type rmap(const scalar_type* alpha, const matrix_type& A, const scalar_type* beta, char transA = 'N',
                   char transB = 'T', const range_type idx = range_type(0, 0)) {
    (void)idx;  // the reference's dense rmap takes the whole map
    return dense_product(false, *alpha, A, *beta, transA, transB, range_type(0, 0));
  }
  // lmap / rmap of a CRS operand, with each map kind's own rules (below).
  matrix_type lmap(const scalar_type* alpha, const crs_matrix_type& B, const scalar_type* beta, char transA = 'N',
                   char transB = 'N', const range_type idx = range_type(0, 0)) {
    return static_cast<Derived*>(this)->lmap_crs(*alpha, B, *beta, transA, transB, idx);
  }
  matrix_type rmap(const scalar_type* alpha, const crs_matrix_type& A, const scalar_type* beta, char transA = 'N',
                   char transB = 'T', const range_type idx = range_type(0, 0)) {
    return static_cast<Derived*>(this)->rmap_crs(*alpha, A, *beta, transA, transB, idx);
  }

  bool issparse() const { return KIND == SKEMA_MAP_SPARSE_SIGN; }
  size_type nrows() const { return nrow; }
  size_type ncols() const { return ncol; }
  // The stored map: Gauss values (nrow x ncol column-major) or SparseSign
  // zeta entries per stored row (values, indices).
  void export_map(std::vector<double>& values, std::vector<int32_t>& indices) const {
    const int z = KIND == SKEMA_MAP_SPARSE_SIGN ? (int)std::max<size_type>(2, std::min<size_type>(ncol, 8)) : 0;
    values.assign(KIND == SKEMA_MAP_SPARSE_SIGN ? nrow * z : nrow * ncol, 0.0);
    indices.assign(KIND == SKEMA_MAP_SPARSE_SIGN ? nrow * z : 0, 0);
    detail::check(skema_dimredux_export(map_.get(), values.data(), indices.empty() ? nullptr : indices.data()),
                  skema_dimredux_last_error(map_.get()));
  }

  DimReduxStats stats;

 protected:
  struct Free {
    void operator()(skema_dimredux* h) const { skema_dimredux_destroy(h); }
  };
  const size_type nrow, ncol;
  const ordinal_type seed;
  const std::string label;
  const bool debug;
  const std::filesystem::path debug_filename;
  const bool init_transposed;
  std::shared_ptr<skema_dimredux> map_;

  // C = alpha op(M(...)) op(B) (left) or alpha op(B) op(M(...)) (right) for a
  // dense FP64 host operand, through the library in FP32.
  matrix_type dense_product(bool left, double alpha, const matrix_type& X, double beta, char tA, char tB,
                            range_type idx) {
    const auto t0 = std::chrono::steady_clock::now();
    const bool tm = left ? (tA == 'T' || tA == 't') : (tB == 'T' || tB == 't');
    const bool tx = left ? (tB == 'T' || tB == 't') : (tA == 'T' || tA == 't');
    const size_type span = idx.first != idx.second ? idx.second - idx.first : (left ? ncol : nrow);
    const size_type mr = left ? nrow : span, mc = left ? span : ncol;  // M restricted
    const size_type om = tm ? mc : mr, on = tm ? mr : mc;               // op(M)
    const size_type xm = tx ? X.extent(1) : X.extent(0), xn = tx ? X.extent(0) : X.extent(1);
    const size_type cm = left ? om : xm, cn = left ? xn : on;
    std::vector<float> xf = detail::to_f32(X), cf(cm * cn, 0.f);
    skema_matf xd{xf.data(), (int64_t)X.extent(0), (int64_t)X.extent(1),
                  (int64_t)std::max<size_type>(1, X.extent(0)), SKEMA_COL_MAJOR};
    skema_matf cd{cf.data(), (int64_t)cm, (int64_t)cn, (int64_t)std::max<size_type>(1, cm), SKEMA_COL_MAJOR};
    const int st = left ? skema_dimredux_lmap(map_.get(), alpha, &xd, beta, tA, tB, (int64_t)idx.first,
                                              (int64_t)idx.second, &cd, SKEMA_MEM_HOST)
                        : skema_dimredux_rmap(map_.get(), alpha, &xd, beta, tA, tB, (int64_t)idx.first,
                                              (int64_t)idx.second, &cd, SKEMA_MEM_HOST);
    detail::check(st, skema_dimredux_last_error(map_.get()));
    stats.map = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return detail::from_f32(cf, cm, cn, label + "::map::C");
  }

  // C = alpha op(M(...)) op(S) (left) or alpha op(S) op(M(...)) (right) for a
  // CRS operand S.
  matrix_type crs_product(bool left, double alpha, const crs_matrix_type& S, double beta, char tA, char tB,
                          range_type idx) {
    const auto t0 = std::chrono::steady_clock::now();
    const bool tm = left ? (tA == 'T' || tA == 't') : (tB == 'T' || tB == 't');
    const bool ts = left ? (tB == 'T' || tB == 't') : (tA == 'T' || tA == 't');
    const size_type span = idx.first != idx.second ? idx.second - idx.first : (left ? ncol : nrow);
    const size_type mr = left ? nrow : span, mc = left ? span : ncol;
    const size_type om = tm ? mc : mr, on = tm ? mr : mc;
    const size_type sm = ts ? S.numCols() : S.numRows(), sn = ts ? S.numRows() : S.numCols();
    const size_type cm = left ? om : sm, cn = left ? sn : on;
    detail::CsrF32 s = detail::to_f32(S);
    std::vector<float> cf(cm * cn, 0.f);
    skema_csrf sd{s.rowptr.data(), s.col.data(), s.val.data(), (int64_t)S.numRows(), (int64_t)S.numCols()};
    skema_matf cd{cf.data(), (int64_t)cm, (int64_t)cn, (int64_t)std::max<size_type>(1, cm), SKEMA_COL_MAJOR};
    const int st = left ? skema_dimredux_lmap_csr(map_.get(), alpha, &sd, beta, tA, tB, (int64_t)idx.first,
                                                  (int64_t)idx.second, &cd, SKEMA_MEM_HOST)
                        : skema_dimredux_rmap_csr(map_.get(), alpha, &sd, beta, tA, tB, (int64_t)idx.first,
                                                  (int64_t)idx.second, &cd, SKEMA_MEM_HOST);
    detail::check(st, skema_dimredux_last_error(map_.get()));
    stats.map = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return detail::from_f32(cf, cm, cn, label + "::map::C");
  }
};

class GaussDimRedux : public DimRedux<GaussDimRedux, SKEMA_MAP_GAUSS> {
 public:
  GaussDimRedux(const size_type nrow_, const size_type ncol_, const ordinal_type seed_,
                const std::string label_ = "GaussDimRedux", const bool debug_ = false,
                const std::filesystem::path debug_filename_ = "", const bool init_transposed_ = false)
      : DimRedux(nrow_, ncol_, seed_, label_, debug_, debug_filename_, init_transposed_) {}
  // CRS lmap (src/Skema_DimRedux_Gauss.cpp:54-76): spmv of op(B) with the
  // map's columns idx, returned transposed: (op(B) M(:, idx))^T; transA is
  // not used (the reference passes it where spmv ignores it).
  matrix_type lmap_crs(double alpha, const crs_matrix_type& B, double beta, char, char transB, range_type idx) {
    const char tb = (transB == 'N' || transB == 'n') ? 'T' : 'N';
    return crs_product(true, alpha, B, beta, 'T', tb, idx);
  }
  // CRS rmap (src/Skema_DimRedux_Gauss.cpp:78-99): op(A) M(idx, :); transB
  // is not used.
  matrix_type rmap_crs(double alpha, const crs_matrix_type& A, double beta, char transA, char, range_type idx) {
    return crs_product(false, alpha, A, beta, transA, 'N', idx);
  }
};

class SparseSignDimRedux : public DimRedux<SparseSignDimRedux, SKEMA_MAP_SPARSE_SIGN> {
 public:
  SparseSignDimRedux(const size_type nrow_, const size_type ncol_, const ordinal_type seed_,
                     const std::string label_ = "SparseSignDimRedux", const bool debug_ = false,
                     const std::filesystem::path debug_filename_ = "", const bool init_transposed_ = false)
      : DimRedux(nrow_, ncol_, seed_, label_, debug_, debug_filename_, init_transposed_) {}
  // CRS lmap / rmap (src/Skema_DimRedux_SparseSign.cpp:53-111): the sparse
  // product M(:, idx) B, resp. A M, densified; the reference's spgemm takes
  // neither alpha nor the transposes, so neither does this.
  matrix_type lmap_crs(double, const crs_matrix_type& B, double, char, char, range_type idx) {
    return crs_product(true, 1.0, B, 0.0, 'N', 'N', idx);
  }
  matrix_type rmap_crs(double, const crs_matrix_type& A, double, char, char, range_type) {
    return crs_product(false, 1.0, A, 0.0, 'N', 'N', range_type(0, 0));
  }
};

// ---- SketchySVD / SketchySPD (src/Skema_SketchySVD.hpp:11-108) ------------
namespace detail {

// One library context over A, owned.
class Context {
 public:
  Context(const AlgParams& p, int32_t kind, bool spd) : alg_(p), spd_(spd) {
    const skema_params cp = p.to_c(kind, spd);
    skema_ctx* c = nullptr;
    const int st = skema_create(&cp, &c);
    if (st != SKEMA_OK) check(st, skema_last_error(nullptr));
    ctx_.reset(c);
    int64_t k = 0, s = 0;
    check_ctx(skema_get_dims(c, &k, &s, nullptr), c);
    range_ = (size_type)k;
    core_ = (size_type)s;
  }
  skema_ctx* get() const { return ctx_.get(); }
  size_type range() const { return range_; }
  size_type core() const { return core_; }

  // Rows [r0, r0 + nr) of A into the sketches (update), or into an open
  // residual pass (residual).
  void stream(const matrix_type& A, size_type r0, size_type nr, bool residual) {
    skema_ctx* c = get();
    if (alg_.kernel_func == Kernel_Map::GAUSSRBF) {
      // A holds the kernel's points, N x d (src/Skema_Window.hpp:90-107)
      const std::vector<float> f = to_f32(A);
      const int64_t N = (int64_t)A.extent(0), d = (int64_t)A.extent(1);
      const int st = residual ? skema_residuals_update_rbf(c, f.data(), N, SKEMA_COL_MAJOR, N, d, (int64_t)r0,
                                                           (int64_t)nr, SKEMA_MEM_HOST)
                              : skema_linear_update_rbf(c, f.data(), N, SKEMA_COL_MAJOR, N, d, (int64_t)r0,
                                                        (int64_t)nr, SKEMA_MEM_HOST);
      check_ctx(st, c);
      return;
    }
    const size_type m = A.extent(0), n = A.extent(1);
    std::vector<float> f(nr * n);
    for (size_type j = 0; j < n; ++j)
      for (size_type i = 0; i < nr; ++i) f[i + j * nr] = (float)A(r0 + i, j);
    const int st = residual ? skema_residuals_update_dense(c, f.data(), (int64_t)std::max<size_type>(nr, 1),
                                                           SKEMA_COL_MAJOR, (int64_t)r0, (int64_t)nr, SKEMA_MEM_HOST)
                            : skema_linear_update_dense(c, f.data(), (int64_t)std::max<size_type>(nr, 1),
                                                        SKEMA_COL_MAJOR, (int64_t)r0, (int64_t)nr, SKEMA_MEM_HOST);
    (void)m;
    check_ctx(st, c);
  }
  void stream(const crs_matrix_type& A, size_type r0, size_type nr, bool residual) {
    skema_ctx* c = get();
    std::vector<int64_t> rp(A.row_map.begin() + r0, A.row_map.begin() + r0 + nr + 1);
    std::vector<int32_t> col(A.entries.begin(), A.entries.end());
    std::vector<float> val(A.values.size());
    for (std::size_t i = 0; i < val.size(); ++i) val[i] = (float)A.values[i];
    const int st = residual ? skema_residuals_update_csr(c, rp.data(), col.data(), val.data(), (int64_t)r0,
                                                         (int64_t)nr, SKEMA_MEM_HOST)
                            : skema_linear_update_csr(c, rp.data(), col.data(), val.data(), (int64_t)r0,
                                                      (int64_t)nr, SKEMA_MEM_HOST);
    check_ctx(st, c);
  }
  static size_type rows_of(const matrix_type& A) { return A.extent(0); }
  static size_type rows_of(const crs_matrix_type& A) { return A.numRows(); }

  // The context's maps as the reference's --debug-file dumps, in their
  // stored orientation (SketchySPD: Omega only).
  void dump_maps(const std::string& stem) const {
    static const std::pair<int32_t, const char*> maps[4] = {
        {SKEMA_UPSILON, "Upsilon"}, {SKEMA_OMEGA, "Omega"}, {SKEMA_PHI, "Phi"}, {SKEMA_PSI, "Psi"}};
    for (const auto& [which, label] : maps) {
      if (spd_ && which != SKEMA_OMEGA) continue;
      int64_t nr = 0, nc = 0;
      int32_t z = 0, tr = 0;
      check_ctx(skema_map_info(get(), which, &nr, &nc, &z, &tr), get());
      std::vector<double> v((size_t)(z ? nr * z : nr * nc));
      std::vector<int32_t> ix((size_t)(z ? nr * z : 0));
      check_ctx(skema_map_export(get(), which, v.data(), z ? ix.data() : nullptr), get());
      write_map_dump(stem, label, nr, nc, z, v, ix);
    }
  }

 private:
  struct Free {
    void operator()(skema_ctx* c) const { skema_destroy(c); }
  };
  AlgParams alg_;
  bool spd_;
  std::unique_ptr<skema_ctx, Free> ctx_;
  size_type range_ = 0, core_ = 0;
};

using Timings = std::map<std::string, std::map<std::string, scalar_type>>;
using Traces = std::map<std::string, std::map<std::string, std::vector<scalar_type>>>;

// The JSON of save_history (src/Skema_SketchySVD.cpp:730-755): keys in
// sorted order (rnrms, svals, timings, traces), four-space indent.
inline void write_history(const std::filesystem::path& fname, const std::vector<double>& svals,
                          const std::vector<double>& rnrms, const Timings& timings, const Traces& traces) {
  std::string o = "{\n";
  auto arr = [](const std::vector<double>& v, const std::string& ind) {
    if (v.empty()) return std::string("[]");
    std::string s = "[\n";
    for (std::size_t i = 0; i < v.size(); ++i) s += ind + "    " + num(v[i]) + (i + 1 < v.size() ? ",\n" : "\n");
    return s + ind + "]";
  };
  o += "    \"rnrms\": " + arr(rnrms, "    ") + ",\n";
  o += "    \"svals\": " + arr(svals, "    ") + ",\n";
  o += "    \"timings\": {";
  std::size_t a = 0;
  for (const auto& [k, inner] : timings) {
    o += std::string(a++ ? "," : "") + "\n        \"" + k + "\": {";
    std::size_t b = 0;
    for (const auto& [kk, v] : inner) o += std::string(b++ ? "," : "") + "\n            \"" + kk + "\": " + num(v);
    o += inner.empty() ? "}" : "\n        }";
  }
  o += timings.empty() ? "},\n" : "\n    },\n";
  o += "    \"traces\": {";
  a = 0;
  for (const auto& [k, inner] : traces) {
    o += std::string(a++ ? "," : "") + "\n        \"" + k + "\": {";
    std::size_t b = 0;
    for (const auto& [kk, v] : inner)
      o += std::string(b++ ? "," : "") + "\n            \"" + kk + "\": " + arr(v, "            ");
    o += inner.empty() ? "}" : "\n        }";
  }
  o += traces.empty() ? "}\n}" : "\n    }\n}";
  if (!fname.filename().empty()) {
    std::ofstream f(fname.filename());
    f << o << std::endl;
  } else {
    std::cout << o << std::endl;
  }
}

// The reference's timing keys (src/Skema_SketchySVD.cpp:101-116 for
// SketchySVD, :776-786 for SketchySPD), in seconds, from the library's
// device stage timers; zero where no stage corresponds or none ran. For
// SketchySVD: update.{upsilon, omega, phi, psi, window, daxpy} from the
// stages of the same names (the sparse-sign X / Z entry kernel counted under
// upsilon, the fused tensor-core window kernel under omega), and
// approx.{dgeqrf, dgels, dgesvd, dgemm} from approx.{orth, core, svd,
// vectors}; the approximations taken for per-window traces are included.
// For SketchySPD: update.{omega, window, daxpy}.
inline Timings reference_timings(skema_ctx* c, bool spd) {
  auto sec = [c](const char* stage) {
    double ms = 0.0;
    int64_t n = 0;
    return skema_timing_get(c, stage, &ms, &n) == SKEMA_OK ? ms / 1e3 : 0.0;
  };
  Timings t;
  if (spd) {
    t["init"]["omega"] = 0.0;
    t["update"]["omega"] = sec("update.omega") + sec("update.fused");
    t["update"]["window"] = sec("update.window");
    t["update"]["daxpy"] = sec("update.daxpy");
    for (const char* k : {"omega", "daxpy", "norm2", "update", "dpotrf", "dgels", "dgesvd"}) t["approx"][k] = 0.0;
    return t;
  }
  for (const char* k : {"upsilon", "omega", "phi", "psi"}) t["init"][k] = 0.0;
  t["update"]["upsilon"] = sec("update.upsilon") + sec("update.entries");
  t["update"]["omega"] = sec("update.omega") + sec("update.fused");
  t["update"]["phi"] = sec("update.phi");
  t["update"]["psi"] = sec("update.psi");
  t["update"]["window"] = sec("update.window");
  t["update"]["daxpy"] = sec("update.daxpy");
  t["approx"]["phi"] = 0.0;
  t["approx"]["psi"] = 0.0;
  t["approx"]["dgeqrf"] = sec("approx.orth");
  t["approx"]["dgels"] = sec("approx.core");
  t["approx"]["dgesvd"] = sec("approx.svd");
  t["approx"]["dgemm"] = sec("approx.vectors");
  return t;
}

inline double seconds_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace detail

template <typename MatrixType, typename DimReduxT>
class SketchySVD {
 public:
  explicit SketchySVD(const AlgParams& p)
      : nrow(p.matrix_m), ncol(p.matrix_n), rank(p.rank), eta(p.sketch_eta), nu(p.sketch_nu), algParams(p),
        ctx_(p, DimReduxT::kind, false), range(ctx_.range()), core(ctx_.core()) {
    detail::check_ctx(skema_timing_enable(ctx_.get(), 1), ctx_.get());  // the reference always times
    // the last approximation's U, S, V stay on the device for compute_residuals
    detail::check_ctx(skema_set_keep_factors(ctx_.get(), 1), ctx_.get());
    if (!p.debug_filename.empty()) ctx_.dump_maps(detail::debug_stem(p.debug_filename));
  }

  // SketchySVD::linear_update (src/Skema_SketchySVD.cpp:120-246): zero the
  // sketches, stream every row window; with sketch_compute_svals_iters the
  // top-rank singular values after each window go to the traces. With
  // --debug-file the sketches are written after every window
  // (<stem>_X.txt.<w>, _Y.txt.<w>, _Z.txt.<w>) and at the end (<stem>_X.txt,
  // ...), as src/Skema_SketchySVD.cpp:191-205, 235-245 write them; a single
  // window of all rows writes none, as the reference returns first.
  void linear_update(const MatrixType& A) {
    skema_ctx* c = ctx_.get();
    detail::check_ctx(skema_reset(c), c);
    const size_type m = algParams.kernel_func == Kernel_Map::GAUSSRBF ? nrow : detail::Context::rows_of(A);
    const size_type W = std::max<size_type>(1, algParams.window);
    const std::string stem = W < m ? detail::debug_stem(algParams.debug_filename) : std::string();
    if (W >= m || (!algParams.sketch_compute_svals_iters && stem.empty())) {
      ctx_.stream(A, 0, m, false);
    } else {
      for (size_type r0 = 0, w = 0; r0 < m; r0 += W, ++w) {
        ctx_.stream(A, r0, std::min(W, m - r0), false);
        if (!stem.empty()) dump_sketches(stem, "." + std::to_string(w));
        if (algParams.sketch_compute_svals_iters) {
          const auto S = std::get<1>(low_rank_approx(false));
          std::vector<double> sv(S.data(), S.data() + S.extent(0));
          traces[std::to_string(w)]["svals"] = sv;
        }
      }
    }
    if (!stem.empty()) dump_sketches(stem, "");
    detail::check_ctx(skema_synchronize(c), c);
  }

  // SketchySVD::low_rank_approx (src/Skema_SketchySVD.cpp:569-664): U (m x r),
  // S (r), V (n x r), FP64.
  std::tuple<matrix_type, vector_type, matrix_type> low_rank_approx(bool update_timers = true) {
    skema_ctx* c = ctx_.get();
    matrix_type U("U", nrow, rank), V("V", ncol, rank);
    vector_type S("S", rank);
    detail::check_ctx(skema_low_rank_approx(c, U.data(), S.data(), V.data(), SKEMA_MEM_HOST), c);
    if (update_timers) {
      uvecs = U;
      svals = S;
      vvecs = V;
    }
    return {U, S, V};
  }

  // SketchySVD::compute_residuals (src/Skema_SketchySVD.cpp:719-727).
  void compute_residuals(const MatrixType& A) {
    const auto t0 = std::chrono::steady_clock::now();
    skema_ctx* c = ctx_.get();
    if (svals.extent(0) == 0) throw std::runtime_error("skema: compute_residuals needs a low_rank_approx first");
    // the factors kept on the device, else (replaced since) the stored ones
    if (skema_residuals_begin(c, nullptr, nullptr, nullptr, SKEMA_MEM_HOST) != SKEMA_OK)
      detail::check_ctx(skema_residuals_begin(c, uvecs.data(), svals.data(), vvecs.data(), SKEMA_MEM_HOST), c);
    const size_type m = algParams.kernel_func == Kernel_Map::GAUSSRBF ? nrow : detail::Context::rows_of(A);
    ctx_.stream(A, 0, m, true);
    rnrms = vector_type("rnrms", rank);
    detail::check_ctx(skema_residuals_finish(c, rnrms.data(), SKEMA_MEM_HOST), c);
    std::cout << "\nCompute residuals: " << detail::seconds_since(t0) << std::endl;
  }

  // SketchySVD::save_history (src/Skema_SketchySVD.cpp:730-755).
  void save_history(std::filesystem::path fname) {
    std::vector<double> s(rank, 0.0), r(rank, 0.0);
    for (size_type i = 0; i < rank; ++i) {
      if (svals.extent(0) > i) s[i] = svals(i);
      if (rnrms.extent(0) > i) r[i] = rnrms(i);
    }
    detail::write_history(fname, s, r, detail::reference_timings(ctx_.get(), false), traces);
  }

  // The sketches (X k x n, Y m x k, Z s x s), FP32 from the device.
  matrix_type sketch(int32_t which) const {
    const size_type rows = which == SKEMA_SKETCH_X ? range : which == SKEMA_SKETCH_Y ? nrow : core;
    const size_type cols = which == SKEMA_SKETCH_X ? ncol : which == SKEMA_SKETCH_Y ? range : core;
    std::vector<float> f(rows * cols);
    detail::check_ctx(skema_get_sketch(ctx_.get(), which, f.data(), (int64_t)std::max<size_type>(rows, 1),
                                       SKEMA_COL_MAJOR, SKEMA_MEM_HOST),
                      ctx_.get());
    return detail::from_f32(f, rows, cols, "sketch");
  }
  skema_ctx* context() const { return ctx_.get(); }

 private:
  void dump_sketches(const std::string& stem, const std::string& suffix) const {
    detail::write_text(stem + "_X.txt" + suffix, sketch(SKEMA_SKETCH_X));
    detail::write_text(stem + "_Y.txt" + suffix, sketch(SKEMA_SKETCH_Y));
    detail::write_text(stem + "_Z.txt" + suffix, sketch(SKEMA_SKETCH_Z));
  }

  const size_type nrow, ncol, rank;
  const scalar_type eta, nu;
  const AlgParams algParams;
  detail::Context ctx_;
  const size_type range, core;
  matrix_type uvecs, vvecs;
  vector_type svals, rnrms;
  detail::Traces traces;
};

template <typename MatrixType, typename DimReduxT>
class SketchySPD {
 public:
  explicit SketchySPD(const AlgParams& p)
      : nrow(p.matrix_m), ncol(p.matrix_n), rank(p.rank), algParams(p), ctx_(p, DimReduxT::kind, true),
        range(ctx_.range()) {
    detail::check_ctx(skema_timing_enable(ctx_.get(), 1), ctx_.get());
    detail::check_ctx(skema_set_keep_factors(ctx_.get(), 1), ctx_.get());
    if (!p.debug_filename.empty()) ctx_.dump_maps(detail::debug_stem(p.debug_filename));
  }

  // SketchySPD::linear_update (src/Skema_SketchySVD.cpp:790-886); with
  // --debug-file, Y is written to <stem>_Y.txt at the end (:880-885), except
  // for a single window of all rows.
  void linear_update(const MatrixType& A) {
    skema_ctx* c = ctx_.get();
    detail::check_ctx(skema_reset(c), c);
    const size_type m = algParams.kernel_func == Kernel_Map::GAUSSRBF ? nrow : detail::Context::rows_of(A);
    ctx_.stream(A, 0, m, false);
    detail::check_ctx(skema_synchronize(c), c);
    if (!algParams.debug_filename.empty() && std::max<size_type>(1, algParams.window) < m)
      detail::write_text(detail::debug_stem(algParams.debug_filename) + "_Y.txt", sketch());
  }

  // The sketch Y (m x k), FP32 from the device.
  matrix_type sketch() const {
    std::vector<float> f(nrow * range);
    detail::check_ctx(skema_get_sketch(ctx_.get(), SKEMA_SKETCH_Y, f.data(), (int64_t)std::max<size_type>(nrow, 1),
                                       SKEMA_COL_MAJOR, SKEMA_MEM_HOST),
                      ctx_.get());
    return detail::from_f32(f, nrow, range, "sketch");
  }

  // SketchySPD::low_rank_approx (src/Skema_SketchySVD.cpp:935-1151): the
  // eigenvectors U (m x r) and eigenvalues S, per AlgParams::spd_approx.
  std::tuple<matrix_type, vector_type> low_rank_approx(bool update_timers = true) {
    skema_ctx* c = ctx_.get();
    matrix_type U("U", nrow, rank);
    vector_type S("S", rank);
    detail::check_ctx(skema_low_rank_approx(c, U.data(), S.data(), nullptr, SKEMA_MEM_HOST), c);
    if (update_timers) {
      uvecs = U;
      svals = S;
    }
    return {U, S};
  }

  // SketchySPD::compute_residuals (src/Skema_SketchySVD.cpp:1206-1213).
  void compute_residuals(const MatrixType& A) {
    const auto t0 = std::chrono::steady_clock::now();
    skema_ctx* c = ctx_.get();
    if (svals.extent(0) == 0) throw std::runtime_error("skema: compute_residuals needs a low_rank_approx first");
    if (skema_residuals_begin(c, nullptr, nullptr, nullptr, SKEMA_MEM_HOST) != SKEMA_OK)
      detail::check_ctx(skema_residuals_begin(c, nullptr, svals.data(), uvecs.data(), SKEMA_MEM_HOST), c);
    const size_type m = algParams.kernel_func == Kernel_Map::GAUSSRBF ? nrow : detail::Context::rows_of(A);
    ctx_.stream(A, 0, m, true);
    rnrms = vector_type("rnrms", rank);
    detail::check_ctx(skema_residuals_finish(c, rnrms.data(), SKEMA_MEM_HOST), c);
    std::cout << "\nCompute residuals: " << detail::seconds_since(t0) << std::endl;
  }

  void save_history(std::filesystem::path fname) {
    std::vector<double> s(rank, 0.0), r(rank, 0.0);
    for (size_type i = 0; i < rank; ++i) {
      if (svals.extent(0) > i) s[i] = svals(i);
      if (rnrms.extent(0) > i) r[i] = rnrms(i);
    }
    detail::write_history(fname, s, r, detail::reference_timings(ctx_.get(), true), detail::Traces{});
  }

 private:
  const size_type nrow, ncol, rank;
  const AlgParams algParams;
  detail::Context ctx_;
  const size_type range;
  matrix_type uvecs;
  vector_type svals, rnrms;
};

// ---- the driver entry (src/Skema_SketchySVD.cpp:1244-1577) ---------------
namespace detail {
template <typename Sketch, typename MatrixType>
void run_three(const MatrixType& matrix, const AlgParams& algParams, matrix_type& U, vector_type& S,
               matrix_type& V) {
  Sketch sketch(algParams);
  try {
    sketch.linear_update(matrix);
  } catch (const std::exception& e) {
    std::cout << "Skema::sketchysvd::linear_update encountered an exception: " << e.what() << std::endl;
    std::exit(EXIT_FAILURE);
  }
  try {
    std::tie(U, S, V) = sketch.low_rank_approx();
  } catch (const std::exception& e) {
    std::cout << "Skema::sketchysvd::low_rank_approx encountered an exception: " << e.what() << std::endl;
    std::exit(EXIT_FAILURE);
  }
  try {
    sketch.compute_residuals(matrix);
  } catch (const std::exception& e) {
    std::cout << "Skema::sketchysvd::compute_residuals encountered an exception: " << e.what() << std::endl;
    std::exit(EXIT_FAILURE);
  }
  if (!algParams.history_filename.empty()) sketch.save_history(algParams.history_filename);
}

template <typename Sketch, typename MatrixType>
void run_spd(const MatrixType& matrix, const AlgParams& algParams, matrix_type& U, vector_type& S) {
  Sketch sketch(algParams);
  try {
    sketch.linear_update(matrix);
  } catch (const std::exception& e) {
    std::cout << "Skema::sketchyspd::linear_update encountered an exception: " << e.what() << std::endl;
    std::exit(EXIT_FAILURE);
  }
  try {
    std::tie(U, S) = sketch.low_rank_approx();
  } catch (const std::exception& e) {
    std::cout << "Skema::sketchyspd::low_rank_approx encountered an exception: " << e.what() << std::endl;
    std::exit(EXIT_FAILURE);
  }
  try {
    sketch.compute_residuals(matrix);
  } catch (const std::exception& e) {
    std::cout << "Skema::sketchyspd::compute_residuals encountered an exception: " << e.what() << std::endl;
    std::exit(EXIT_FAILURE);
  }
  if (!algParams.history_filename.empty()) sketch.save_history(algParams.history_filename);
}

}  // namespace detail

// Skema::sketchysvd: update, fixed-rank approximation, residuals and the
// history file; SketchySPD when issymmetric without force_three_sketch. The
// results (U, S, V) are also returned (the reference only writes them with
// --debug-file, as here).
template <typename MatrixType>
std::tuple<matrix_type, vector_type, matrix_type> sketchysvd(const MatrixType& matrix, const AlgParams& algParams) {
  matrix_type U, V;
  vector_type S;
  const bool spd = algParams.issymmetric && !algParams.force_three_sketch;
  if (algParams.dim_redux == DimRedux_Map::GAUSS) {
    if (spd)
      detail::run_spd<SketchySPD<MatrixType, GaussDimRedux>>(matrix, algParams, U, S);
    else
      detail::run_three<SketchySVD<MatrixType, GaussDimRedux>>(matrix, algParams, U, S, V);
  } else if (algParams.dim_redux == DimRedux_Map::SPARSE_SIGN) {
    if (spd)
      detail::run_spd<SketchySPD<MatrixType, SparseSignDimRedux>>(matrix, algParams, U, S);
    else
      detail::run_three<SketchySVD<MatrixType, SparseSignDimRedux>>(matrix, algParams, U, S, V);
  } else {
    std::cout << "DimRedux: make another selection." << std::endl;
    std::exit(1);
  }
  if (!algParams.debug_filename.empty()) {
    const std::string stem = algParams.debug_filename.filename().stem().string();
    if (U.extent(0) > 0 && U.extent(1) > 0) detail::write_text(stem + "_U.txt", U);
    if (S.extent(0) > 0) detail::write_text(stem + "_S.txt", S);
    if (V.extent(0) > 0 && V.extent(1) > 0) detail::write_text(stem + "_V.txt", V);
  }
  return {U, S, V};
}

}  // namespace Skema

#endif  // SKEMA_HPP
