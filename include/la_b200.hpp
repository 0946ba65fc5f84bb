// la_b200.hpp -- header-only C++ drop-in for the reference's hot-path API.
//
// Same class and function names, template parameters and call signatures
// as the reference's sparse_mat_op/ headers, in namespace
// matrix_utils::b200, forwarding to the C-ABI in la_b200.h (the GPU does
// the work).  A caller switches by replacing
//     matrix_utils::SegSumSPMV<int, int, double>
// with
//     matrix_utils::b200::SegSumSPMV<int, int, double>
// (and likewise ALBUSSPMV, SPMV, OptimizedTriangularSolve,
// TopologicalSort2).  Only the <int, int, double> instantiation exists, as
// in the reference (triangle_solve.cpp:3-44, precond.cpp:4-27).
//
// Semantics kept: preprocess()/analysis() run once per matrix and the matrix
// must not change afterwards (the reference's preprocessed state assumes the
// same); operator() is const but uses the object's device scratch, so one
// object must not be called from two threads at once.  Differences: b and x
// are host arrays here as in the reference, and each call copies b in and x
// out (use the C-ABI device-pointer entry points to keep vectors resident);
// when beta == 0, x is not read.  Errors throw matrix_utils::b200::Error.
#pragma once

#include "la_b200.h"

#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

namespace matrix_utils {
namespace b200 {

struct Error : std::runtime_error {
  la_status status;
  Error(la_status s, const std::string &what)
      : std::runtime_error(what + ": " + la_last_error_string()), status(s) {}
};

inline void check(la_status s, const char *what) {
  if (s != LA_OK)
    throw Error(s, what);
}

template <typename R, typename C, typename V> constexpr void require_int_double() {
  static_assert(std::is_same_v<R, int> && std::is_same_v<C, int> &&
                    std::is_same_v<V, double>,
                "only the <int, int, double> instantiation is provided, as in "
                "the reference");
}

// SegSumSPMV (spmv.hpp:59-185) / ALBUSSPMV (spmv.hpp:186-300).
template <la_spmv_kind KIND, typename ROWTYPE = int, typename COLTYPE = int,
          typename VALTYPE = double>
class SpmvGpu {
public:
  explicit SpmvGpu(const int num_threads = 1) : _nthreads{num_threads} {
    require_int_double<ROWTYPE, COLTYPE, VALTYPE>();
  }
  ~SpmvGpu() { release(); }
  SpmvGpu(const SpmvGpu &) = delete;
  SpmvGpu &operator=(const SpmvGpu &) = delete;

  void setNumThreads(const int num_threads) { _nthreads = num_threads; }

  void preprocess(const COLTYPE size, const int base, ROWTYPE const *ai,
                  COLTYPE const *aj, VALTYPE const *av) {
    release();
    COLTYPE ncols = size;
    for (ROWTYPE k = 0; k < ai[size] - base; k++)
      ncols = aj[k] - base + 1 > ncols ? aj[k] - base + 1 : ncols;
    check(la_csr_create(size, ncols, base, ai, aj, av, LA_F64, 0, &_A),
          "la_csr_create");
    check(la_spmv_plan_create(_A, KIND, &_plan), "la_spmv_plan_create");
    _size = size;
  }

  // x = alpha * A * b + beta * x
  void operator()(const COLTYPE size, const int base, ROWTYPE const *ai,
                  COLTYPE const *aj, VALTYPE const *av, const VALTYPE *const b,
                  VALTYPE *const x, const VALTYPE alpha,
                  const VALTYPE beta) const {
    if (!_plan || size != _size)
      const_cast<SpmvGpu *>(this)->preprocess(size, base, ai, aj, av);
    check(la_spmv_host(_plan, alpha, b, beta, x), "la_spmv_host");
  }

  int get_num_threads() const { return _nthreads; }

private:
  void release() {
    if (_plan)
      la_spmv_plan_destroy(_plan);
    if (_A)
      la_csr_destroy(_A);
    _plan = nullptr;
    _A = nullptr;
  }
  int _nthreads;
  COLTYPE _size{-1};
  la_csr_t _A{nullptr};
  la_spmv_plan_t _plan{nullptr};
};

template <typename R = int, typename C = int, typename V = double>
using SegSumSPMV = SpmvGpu<LA_SPMV_SEGSUM, R, C, V>;
template <typename R = int, typename C = int, typename V = double>
using ALBUSSPMV = SpmvGpu<LA_SPMV_ALBUS, R, C, V>;

// SPMV<CSRMatrixType, SPMVType> adapter (spmv.hpp:310-334).
template <typename CSRMatrixType, typename SPMVType> struct SPMV {
  using ROWTYPE = typename CSRMatrixType::ROWTYPE;
  using COLTYPE = typename CSRMatrixType::COLTYPE;
  using VALTYPE = typename CSRMatrixType::VALTYPE;

  SPMV() : _matrix{nullptr} {}
  void setMatrix(CSRMatrixType const *matrix) { _matrix = matrix; }
  void preprocess() {
    _spmv.preprocess(_matrix->rows, _matrix->Base(), _matrix->AI(),
                     _matrix->AJ(), _matrix->AV());
  }
  void operator()(const VALTYPE *const b, VALTYPE *const x,
                  const VALTYPE alpha = 1., const VALTYPE beta = 0.) const {
    _spmv(_matrix->rows, _matrix->Base(), _matrix->AI(), _matrix->AJ(),
          _matrix->AV(), b, x, alpha, beta);
  }
  CSRMatrixType const *_matrix;
  SPMVType _spmv;
};

enum TriangularMatrix { L = 0, U = 1 };
enum class FBSubstitutionType { Barrier, NoBarrier, NoBarrierSuperNode };

// OptimizedTriangularSolve (triangle_solve.hpp:149-208).  Every FBST maps to
// the one GPU schedule (persistent kernel, per-row readiness).
template <FBSubstitutionType FBST = FBSubstitutionType::Barrier,
          TriangularMatrix TS = TriangularMatrix::L, typename ROWTYPE = int,
          typename COLTYPE = int, typename VALTYPE = double>
class OptimizedTriangularSolve {
public:
  explicit OptimizedTriangularSolve(const int num_threads = 1)
      : _nthreads{num_threads} {
    require_int_double<ROWTYPE, COLTYPE, VALTYPE>();
  }
  ~OptimizedTriangularSolve() {
    if (_plan)
      la_trsv_plan_destroy(_plan);
  }
  OptimizedTriangularSolve(const OptimizedTriangularSolve &) = delete;
  OptimizedTriangularSolve &operator=(const OptimizedTriangularSolve &) = delete;

  void analysis(const COLTYPE rows, const int base, ROWTYPE const *ai,
                COLTYPE const *aj, VALTYPE const *av,
                VALTYPE const *diag = nullptr) {
    if (_plan)
      la_trsv_plan_destroy(_plan);
    _plan = nullptr;
    check(la_trsv_analysis(TS == L ? LA_LOWER : LA_UPPER, rows, base, ai, aj,
                           av, diag, LA_F64, &_plan),
          "la_trsv_analysis");
  }

  void operator()(const VALTYPE *const b, VALTYPE *const x) const {
    check(la_trsv_host(_plan, b, x), "la_trsv_host");
  }

  int get_num_threads() const { return _nthreads; }

private:
  int _nthreads;
  la_trsv_plan_t _plan{nullptr};
};

// The reference's free solve functions (triangle_solve.hpp:32-145), host
// arrays, same signatures.  Each call plans the triangle on the GPU, solves
// once and releases the plan; for repeated solves keep an
// OptimizedTriangularSolve.  Results are bit-identical to the reference's
// (per row: the sum in stored order, then b - sum, / diag).
namespace detail {
inline void solve_with(la_trsv_plan_t plan, la_status made, const double *b, double *x) {
  check(made, "la_trsv_analysis");
  const la_status s = la_trsv_host(plan, b, x);
  la_trsv_plan_destroy(plan);
  check(s, "la_trsv_host");
}
} // namespace detail

// ForwardSubstitution (triangle_solve.hpp:32-43): unit lower, strict L CSR.
template <typename ROWTYPE, typename COLTYPE, typename VALTYPE>
void ForwardSubstitution(const COLTYPE size, const int base, ROWTYPE const *ai,
                         COLTYPE const *aj, VALTYPE const *av, VALTYPE const *const b,
                         VALTYPE *const x) {
  require_int_double<ROWTYPE, COLTYPE, VALTYPE>();
  la_trsv_plan_t p = nullptr;
  const la_status s = la_trsv_analysis(LA_LOWER, size, base, ai, aj, av, nullptr, LA_F64, &p);
  detail::solve_with(p, s, b, x);
}

// BackwardSubstitution (triangle_solve.hpp:59-71): strict U CSR + diag.
template <typename ROWTYPE, typename COLTYPE, typename VALTYPE>
void BackwardSubstitution(const COLTYPE size, const int base, ROWTYPE const *ai,
                          COLTYPE const *aj, VALTYPE const *av, VALTYPE const *diag,
                          VALTYPE const *const b, VALTYPE *const x) {
  require_int_double<ROWTYPE, COLTYPE, VALTYPE>();
  la_trsv_plan_t p = nullptr;
  const la_status s = la_trsv_analysis(LA_UPPER, size, base, ai, aj, av, diag, LA_F64, &p);
  detail::solve_with(p, s, b, x);
}

// LevelScheduleForward/BackwardSubstitution (triangle_solve.hpp:100-145):
// the caller's level structure (iperm with base, zero-based prefix).
template <typename ROWTYPE, typename COLTYPE, typename VALTYPE>
void LevelScheduleForwardSubstitution(COLTYPE const *iperm, COLTYPE const *prefix,
                                      const COLTYPE lvls, const COLTYPE rows, const int base,
                                      ROWTYPE const *ai, COLTYPE const *aj, VALTYPE const *av,
                                      VALTYPE const *const b, VALTYPE *const x) {
  require_int_double<ROWTYPE, COLTYPE, VALTYPE>();
  la_trsv_plan_t p = nullptr;
  const la_status s = la_trsv_analysis_levels(LA_LOWER, rows, base, ai, aj, av, nullptr,
                                              LA_F64, iperm, prefix, lvls, &p);
  detail::solve_with(p, s, b, x);
}

template <typename ROWTYPE, typename COLTYPE, typename VALTYPE>
void LevelScheduleBackwardSubstitution(COLTYPE const *iperm, COLTYPE const *prefix,
                                       const COLTYPE lvls, const COLTYPE rows, const int base,
                                       ROWTYPE const *ai, COLTYPE const *aj, VALTYPE const *av,
                                       VALTYPE const *diag, VALTYPE const *const b,
                                       VALTYPE *const x) {
  require_int_double<ROWTYPE, COLTYPE, VALTYPE>();
  la_trsv_plan_t p = nullptr;
  const la_status s = la_trsv_analysis_levels(LA_UPPER, rows, base, ai, aj, av, diag,
                                              LA_F64, iperm, prefix, lvls, &p);
  detail::solve_with(p, s, b, x);
}

// ForwardSubstitutionT (triangle_solve.hpp:87-98): x = (I + U^T)^-1 b for the
// strict upper triangle U given as CSR, host arrays.  Plans the transposed
// solve on the GPU (la_trsv_analysis_transposed) and runs it once; FP64
// results agree with the reference's column scatter to rounding.
template <typename ROWTYPE, typename COLTYPE, typename VALTYPE>
void ForwardSubstitutionT(const COLTYPE size, const int base, ROWTYPE const *ai,
                          COLTYPE const *aj, VALTYPE const *av,
                          VALTYPE const *const b, VALTYPE *const x) {
  require_int_double<ROWTYPE, COLTYPE, VALTYPE>();
  la_trsv_plan_t plan = nullptr;
  check(la_trsv_analysis_transposed(LA_UPPER, size, base, ai, aj, av, nullptr, LA_F64, &plan),
        "la_trsv_analysis_transposed");
  const la_status s = la_trsv_host(plan, b, x);
  la_trsv_plan_destroy(plan);
  check(s, "la_trsv_host");
}

// permute / permuteRow / permuteVec (matrix_utils.hpp:429-480, 562-576),
// Diagonal (:677-704) and inversePermute (utils/utils.cpp:101-108): host
// functions, bit-identical to the reference.
template <typename ROWTYPE, typename COLTYPE, typename VALTYPE>
void permute(const COLTYPE rows, const int base, ROWTYPE const *ai, COLTYPE const *aj,
             VALTYPE const *av, COLTYPE const *iperm, COLTYPE const *perm,
             ROWTYPE *permed_ai, COLTYPE *permed_aj, VALTYPE *permed_av) {
  require_int_double<ROWTYPE, COLTYPE, VALTYPE>();
  check(la_permute(rows, base, ai, aj, av, iperm, perm, permed_ai, permed_aj, permed_av),
        "la_permute");
}

template <typename ROWTYPE, typename COLTYPE, typename VALTYPE>
void permuteRow(const COLTYPE rows, const int base, ROWTYPE const *ai, COLTYPE const *aj,
                VALTYPE const *av, COLTYPE const *iperm, ROWTYPE *permed_ai,
                COLTYPE *permed_aj, VALTYPE *permed_av) {
  permute(rows, base, ai, aj, av, iperm, (COLTYPE const *)nullptr, permed_ai, permed_aj,
          permed_av);
}

template <typename COLTYPE, typename VALTYPE>
void permuteVec(const COLTYPE rows, const int base, VALTYPE const *const v,
                COLTYPE const *const iperm, VALTYPE *const permed_v) {
  require_int_double<COLTYPE, COLTYPE, VALTYPE>();
  check(la_permute_vec(rows, base, v, iperm, permed_v), "la_permute_vec");
}

template <typename ROWTYPE, typename COLTYPE, typename VALTYPE>
bool Diagonal(const COLTYPE rows, const int base, ROWTYPE const *ai, COLTYPE const *aj,
              VALTYPE const *av, ROWTYPE *diagpos, VALTYPE *diag, const bool invert = false) {
  require_int_double<ROWTYPE, COLTYPE, VALTYPE>();
  int all = 0;
  check(la_diagonal(rows, base, ai, aj, av, diagpos, diag, invert ? 1 : 0, &all),
        "la_diagonal");
  return all != 0;
}

template <typename VEC>
void inversePermute(VEC &iperm, const VEC &perm, const int base) {
  iperm.resize(perm.size());
  check(la_inverse_permute((int)perm.size(), base, perm.data(), iperm.data()),
        "la_inverse_permute");
}

// TopologicalSort<TS> (matrix_utils.hpp:583-635, Kahn's breadth-first
// order), bit-identical output, including the return value (the last level's
// index) and prefix's length (that + 2).
template <TriangularMatrix TS = L, typename ROWTYPE, typename COLTYPE,
          typename VEC>
COLTYPE TopologicalSort(const COLTYPE nodes, const int base, ROWTYPE const *ai,
                        COLTYPE const *aj, VEC &iperm, VEC &prefix) {
  iperm.resize(nodes);
  prefix.resize(nodes + 2);
  int result = 0;
  check(la_topological_sort(TS == L ? LA_LOWER : LA_UPPER, nodes, base, ai, aj,
                            iperm.data(), prefix.data(), &result),
        "la_topological_sort");
  prefix.resize(result + 2);
  return result;
}

// TopologicalSort2<TS> (matrix_utils.hpp:637-675), bit-identical output.
template <TriangularMatrix TS = L, typename ROWTYPE, typename COLTYPE,
          typename VEC>
COLTYPE TopologicalSort2(const COLTYPE nodes, const int base, ROWTYPE const *ai,
                         COLTYPE const *aj, VEC &iperm, VEC &prefix) {
  iperm.resize(nodes);
  prefix.resize(nodes + 1);
  int levels = 0;
  check(la_topological_sort2(TS == L ? LA_LOWER : LA_UPPER, nodes, base, ai,
                             aj, iperm.data(), prefix.data(), &levels),
        "la_topological_sort2");
  prefix.resize(levels + 1);
  return levels;
}

} // namespace b200
} // namespace matrix_utils

// The file readers of utils/utils.h, in utils::b200 with the reference's
// signatures (a caller switches utils::ReadFromBinaryCSR to
// utils::b200::ReadFromBinaryCSR).  ReadFromBinaryCOO reads on the host;
// ReadFromBinaryCSR and read_matrix_market_csr sort the entries into a CSR on
// the GPU (la_csr_read_binary_coo / la_csr_parse_matrix_market) and return
// host vectors, as the reference's do.
#include <istream>
#include <iterator>
#include <string>
#include <utility>

namespace utils {
namespace b200 {

// ReadFromBinaryCOO (utils.h:23-44): entries in file order; returns
// {largest row + 1 - base, largest column + 1 - base}.
template <typename IVEC, typename VVEC, typename IB>
auto ReadFromBinaryCOO(const std::string &filename, IVEC &rows, IVEC &cols, VVEC &vals,
                       const IB base) {
  long long nnz = 0;
  int m = 0, n = 0;
  matrix_utils::b200::check(la_read_binary_coo(filename.c_str(), (int)base, &nnz, nullptr,
                                               nullptr, nullptr, &m, &n),
                            "la_read_binary_coo");
  std::vector<int> r(nnz), c(nnz);
  std::vector<double> v(nnz);
  matrix_utils::b200::check(la_read_binary_coo(filename.c_str(), (int)base, &nnz, r.data(),
                                               c.data(), v.data(), &m, &n),
                            "la_read_binary_coo");
  rows.assign(r.begin(), r.end());
  cols.assign(c.begin(), c.end());
  vals.assign(v.begin(), v.end());
  using I = typename IVEC::value_type;
  return std::make_pair((I)m, (I)n);
}

namespace detail {
template <typename IVEC, typename VVEC>
void download(la_csr_t A, IVEC &ai, IVEC &aj, VVEC &av) {
  int n = 0, nnz = 0;
  la_csr_info(A, &n, nullptr, &nnz, nullptr, nullptr);
  std::vector<int> a(n + 1), j(nnz);
  std::vector<double> v(nnz);
  const la_status s = la_csr_download(A, a.data(), j.data(), v.data());
  la_csr_destroy(A);
  matrix_utils::b200::check(s, "la_csr_download");
  ai.assign(a.begin(), a.end());
  aj.assign(j.begin(), j.end());
  av.assign(v.begin(), v.end());
}
} // namespace detail

// ReadFromBinaryCSR (utils.h:46-91): rows sorted by (row, col), row pointers
// with the file's base; returns {rows, cols} as ReadFromBinaryCOO does.
template <typename IVEC, typename VVEC, typename IB>
auto ReadFromBinaryCSR(const std::string &filename, IVEC &ai, IVEC &aj, VVEC &av,
                       const IB base) {
  la_csr_t A = nullptr;
  matrix_utils::b200::check(la_csr_read_binary_coo(filename.c_str(), (int)base, 0, &A),
                            "la_csr_read_binary_coo");
  int m = 0, n = 0;
  la_csr_info(A, &m, &n, nullptr, nullptr, nullptr);
  detail::download(A, ai, aj, av);
  using I = typename IVEC::value_type;
  return std::make_pair((I)m, (I)n);
}

// read_matrix_market_csr (utils.h:93-132): a 0-based CSR (rows[nrows+1],
// cols, values) from a Matrix Market coordinate stream.
template <typename IVEC, typename VVEC>
void read_matrix_market_csr(std::istream &instream, IVEC &rows, IVEC &cols, VVEC &values) {
  const std::string text((std::istreambuf_iterator<char>(instream)),
                         std::istreambuf_iterator<char>());
  la_csr_t A = nullptr;
  matrix_utils::b200::check(la_csr_parse_matrix_market(text.data(), text.size(), 0, &A),
                            "la_csr_parse_matrix_market");
  detail::download(A, rows, cols, values);
}

} // namespace b200
} // namespace utils
