// ref_shim.cpp -- TEST INFRASTRUCTURE ONLY (oracle side, never shipped).
//
// A thin extern "C" shim over the reference's OWN hot-path templates, compiled
// in place from the reference source tree by oracle/Makefile into
// oracle/_ref/libla_ref.so.  Nothing here re-implements an algorithm: every
// function forwards to the reference code named in its comment, so that the
// tests can (a) pin the oracle's C restatement (oracle/la_oracle.c) against
// the real reference and (b) time the reference's OpenMP path as the CPU
// baseline.  Only the test suite, __graft_entry__.smoke() and bench.py's
// reference / cpu_baseline legs load this library.
//
// All indices are int32 and values double, the only instantiation the
// reference ships (sparse_mat_op/triangle_solve.cpp:3-44,
// sparse_mat_op/precond.cpp:4-27, sparse_mat_op/matrix_utils.cpp:4-105).

#include "matrix_utils.hpp"
#include "precond.hpp"
#include "spmv.hpp"
#include "triangle_solve.hpp"
#include "Reordering.h"
#include "mkl_sparse_mat.h"
#include "utils.h"

#include <cmath>
#include <cstring>
#include <memory>
#include <omp.h>
#include <vector>

using namespace matrix_utils;

extern "C" {

int la_ref_max_threads(void) { return omp_get_max_threads(); }
void la_ref_set_threads(int t) { omp_set_num_threads(t); }

// LoadPrefixBalancedPartitionPos (utils/utils.h:187-222) over the row
// pointers, as ParallelSPMV calls it: start[t] = first row of part t.
void la_ref_prefix_partition(int n, const int *ai, int nparts, int *start) {
  for (int t = 0; t < nparts; t++)
    start[t] = (int)utils::LoadPrefixBalancedPartitionPos(ai, ai + n, t, nparts).first;
  start[nparts] = n;
}

// ---------------------------------------------------------------- SpMV
// SerialSPMV (sparse_mat_op/spmv.hpp:12-29)
void la_ref_serial_spmv(int n, int base, const int *ai, const int *aj,
                        const double *av, const double *b, double *x,
                        double alpha, double beta) {
  SerialSPMV s;
  s(n, base, ai, aj, av, b, x, alpha, beta);
}

// ParallelSPMV (sparse_mat_op/spmv.hpp:31-57), nthreads OpenMP threads
void la_ref_parallel_spmv(int nthreads, int n, int base, const int *ai,
                          const int *aj, const double *av, const double *b,
                          double *x, double alpha, double beta) {
  omp_set_num_threads(nthreads);
  ParallelSPMV s;
  s(n, base, ai, aj, av, b, x, alpha, beta);
}

// SegSumSPMV (sparse_mat_op/spmv.hpp:59-185): preprocess once, apply many.
void *la_ref_segsum_create(int nthreads, int n, int base, const int *ai,
                           const int *aj, const double *av) {
  auto *s = new SegSumSPMV<int, int, double>(nthreads);
  s->preprocess(n, base, ai, aj, av);
  return s;
}
void la_ref_segsum_apply(void *h, int n, int base, const int *ai, const int *aj,
                         const double *av, const double *b, double *x,
                         double alpha, double beta) {
  (*static_cast<SegSumSPMV<int, int, double> *>(h))(n, base, ai, aj, av, b, x,
                                                     alpha, beta);
}
void la_ref_segsum_destroy(void *h) {
  delete static_cast<SegSumSPMV<int, int, double> *>(h);
}

// ALBUSSPMV (sparse_mat_op/spmv.hpp:186-300)
void *la_ref_albus_create(int nthreads, int n, int base, const int *ai,
                          const int *aj, const double *av) {
  auto *s = new ALBUSSPMV<int, int, double>(nthreads);
  s->preprocess(n, base, ai, aj, av);
  return s;
}
void la_ref_albus_apply(void *h, int n, int base, const int *ai, const int *aj,
                        const double *av, const double *b, double *x,
                        double alpha, double beta) {
  (*static_cast<ALBUSSPMV<int, int, double> *>(h))(n, base, ai, aj, av, b, x,
                                                    alpha, beta);
}
void la_ref_albus_destroy(void *h) {
  delete static_cast<ALBUSSPMV<int, int, double> *>(h);
}

// ------------------------------------------------------- triangular solves
// ForwardSubstitution / BackwardSubstitution / ForwardSubstitutionT
// (sparse_mat_op/triangle_solve.hpp:32-98)
void la_ref_forward_substitution(int n, int base, const int *ai, const int *aj,
                                 const double *av, const double *b, double *x) {
  ForwardSubstitution(n, base, ai, aj, av, b, x);
}
void la_ref_backward_substitution(int n, int base, const int *ai,
                                  const int *aj, const double *av,
                                  const double *diag, const double *b,
                                  double *x) {
  BackwardSubstitution(n, base, ai, aj, av, diag, b, x);
}
void la_ref_forward_substitution_t(int n, int base, const int *ai,
                                   const int *aj, const double *av,
                                   const double *b, double *x) {
  ForwardSubstitutionT(n, base, ai, aj, av, b, x);
}

// LevelScheduleForward/BackwardSubstitution (triangle_solve.hpp:100-145)
void la_ref_level_forward(int nthreads, const int *iperm, const int *prefix,
                          int lvls, int n, int base, const int *ai,
                          const int *aj, const double *av, const double *b,
                          double *x) {
  omp_set_num_threads(nthreads);
  LevelScheduleForwardSubstitution(iperm, prefix, lvls, n, base, ai, aj, av, b,
                                   x);
}
void la_ref_level_backward(int nthreads, const int *iperm, const int *prefix,
                           int lvls, int n, int base, const int *ai,
                           const int *aj, const double *av, const double *diag,
                           const double *b, double *x) {
  omp_set_num_threads(nthreads);
  LevelScheduleBackwardSubstitution(iperm, prefix, lvls, n, base, ai, aj, av,
                                    diag, b, x);
}

// OptimizedTriangularSolve<FBST, L|U> (triangle_solve.hpp:149-208,
// triangle_solve.tpp:17-226).  kind: 0 Barrier, 1 NoBarrier,
// 2 NoBarrierSuperNode.  uplo: 0 L, 1 U.  diag may be null (unit diagonal);
// the reference keeps the pointer, so it must outlive the handle.
struct RefTrsv {
  int kind, uplo;
  void *obj;
};

// ------------------------------------------------------------ file readers
// utils::ReadFromBinaryCOO (utils/utils.h:23-44).  Returns the entry count;
// with rows != NULL the entries (file order) and *m / *n are written too.
long long la_ref_read_binary_coo(const char *path, int base, int *rows, int *cols,
                                 double *vals, int *m, int *n) {
  std::vector<int> r, c;
  std::vector<double> v;
  auto mn = utils::ReadFromBinaryCOO(path, r, c, v, base);
  if (rows) {
    std::memcpy(rows, r.data(), sizeof(int) * r.size());
    std::memcpy(cols, c.data(), sizeof(int) * c.size());
    std::memcpy(vals, v.data(), sizeof(double) * v.size());
  }
  if (m)
    *m = mn.first;
  if (n)
    *n = mn.second;
  return (long long)r.size();
}

// utils::ReadFromBinaryCSR (utils/utils.h:46-91): ai[m + 1], aj / av[nnz].
long long la_ref_read_binary_csr(const char *path, int base, int *ai, int *aj, double *av,
                                 int *m, int *n) {
  std::vector<int> a, j;
  std::vector<double> v;
  auto mn = utils::ReadFromBinaryCSR(path, a, j, v, base);
  if (ai) {
    std::memcpy(ai, a.data(), sizeof(int) * a.size());
    std::memcpy(aj, j.data(), sizeof(int) * j.size());
    std::memcpy(av, v.data(), sizeof(double) * v.size());
  }
  if (m)
    *m = mn.first;
  if (n)
    *n = mn.second;
  return (long long)j.size();
}

} // extern "C"

template <FBSubstitutionType K, TriangularMatrix T>
static void *make_trsv(int nthreads, int n, int base, const int *ai,
                       const int *aj, const double *av, const double *diag) {
  auto *o = new OptimizedTriangularSolve<K, T, int, int, double>(nthreads);
  o->analysis(n, base, ai, aj, av, diag);
  return o;
}

extern "C" {

void *la_ref_trsv_create(int kind, int uplo, int nthreads, int n, int base,
                         const int *ai, const int *aj, const double *av,
                         const double *diag) {
  auto *h = new RefTrsv{kind, uplo, nullptr};
  using F = FBSubstitutionType;
  if (uplo == 0) {
    if (kind == 0) h->obj = make_trsv<F::Barrier, L>(nthreads, n, base, ai, aj, av, diag);
    if (kind == 1) h->obj = make_trsv<F::NoBarrier, L>(nthreads, n, base, ai, aj, av, diag);
    if (kind == 2) h->obj = make_trsv<F::NoBarrierSuperNode, L>(nthreads, n, base, ai, aj, av, diag);
  } else {
    if (kind == 0) h->obj = make_trsv<F::Barrier, U>(nthreads, n, base, ai, aj, av, diag);
    if (kind == 1) h->obj = make_trsv<F::NoBarrier, U>(nthreads, n, base, ai, aj, av, diag);
    if (kind == 2) h->obj = make_trsv<F::NoBarrierSuperNode, U>(nthreads, n, base, ai, aj, av, diag);
  }
  return h;
}

#define LA_REF_TRSV_DISPATCH(EXPR)                                               \
  do {                                                                           \
    using F = FBSubstitutionType;                                                \
    if (h->uplo == 0) {                                                          \
      if (h->kind == 0) { auto *o = static_cast<OptimizedTriangularSolve<F::Barrier, L, int, int, double> *>(h->obj); EXPR; } \
      if (h->kind == 1) { auto *o = static_cast<OptimizedTriangularSolve<F::NoBarrier, L, int, int, double> *>(h->obj); EXPR; } \
      if (h->kind == 2) { auto *o = static_cast<OptimizedTriangularSolve<F::NoBarrierSuperNode, L, int, int, double> *>(h->obj); EXPR; } \
    } else {                                                                     \
      if (h->kind == 0) { auto *o = static_cast<OptimizedTriangularSolve<F::Barrier, U, int, int, double> *>(h->obj); EXPR; } \
      if (h->kind == 1) { auto *o = static_cast<OptimizedTriangularSolve<F::NoBarrier, U, int, int, double> *>(h->obj); EXPR; } \
      if (h->kind == 2) { auto *o = static_cast<OptimizedTriangularSolve<F::NoBarrierSuperNode, U, int, int, double> *>(h->obj); EXPR; } \
    }                                                                            \
  } while (0)

void la_ref_trsv_apply(void *hv, const double *b, double *x) {
  auto *h = static_cast<RefTrsv *>(hv);
  LA_REF_TRSV_DISPATCH((*o)(b, x));
}
void la_ref_trsv_destroy(void *hv) {
  auto *h = static_cast<RefTrsv *>(hv);
  LA_REF_TRSV_DISPATCH(delete o);
  delete h;
}

// ------------------------------------------------------ host preprocessing
// TopologicalSort2<L|U> (matrix_utils.hpp:637-675).  iperm has n entries,
// prefix capacity n + 1; returns the number of levels.
int la_ref_topological_sort2(int uplo, int n, int base, const int *ai,
                             const int *aj, int *iperm, int *prefix) {
  std::vector<int> ip, pf;
  int lv = uplo == 0 ? TopologicalSort2<L>(n, base, ai, aj, ip, pf)
                     : TopologicalSort2<U>(n, base, ai, aj, ip, pf);
  std::memcpy(iperm, ip.data(), sizeof(int) * ip.size());
  std::memcpy(prefix, pf.data(), sizeof(int) * pf.size());
  return lv;
}

// TopologicalSort (Kahn BFS form, matrix_utils.hpp:583-635)
int la_ref_topological_sort(int uplo, int n, int base, const int *ai,
                            const int *aj, int *iperm, int *prefix) {
  std::vector<int> ip, pf;
  int lv = uplo == 0 ? TopologicalSort<L>(n, base, ai, aj, ip, pf)
                     : TopologicalSort<U>(n, base, ai, aj, ip, pf);
  std::memcpy(iperm, ip.data(), sizeof(int) * ip.size());
  std::memcpy(prefix, pf.data(), sizeof(int) * pf.size());
  return lv;
}

// SplitLDU (matrix_utils.hpp:720-803).  Output buffers sized nnz (L, U) and
// n + 1 (row pointers), n (D).  Returns L nnz in *lnnz and U nnz in *unnz.
void la_ref_split_ldu(int n, int base, const int *ai, const int *aj,
                      const double *av, int *l_ai, int *l_aj, double *l_av,
                      double *d, int *u_ai, int *u_aj, double *u_av, int *lnnz,
                      int *unnz) {
  CSRMatrixVec<int, int, double> Lm, Um;
  std::vector<double> D;
  SplitLDU(n, base, ai, aj, av, Lm, D, Um);
  std::memcpy(l_ai, Lm.ai.data(), sizeof(int) * (n + 1));
  std::memcpy(u_ai, Um.ai.data(), sizeof(int) * (n + 1));
  std::memcpy(l_aj, Lm.aj.data(), sizeof(int) * Lm.aj.size());
  std::memcpy(l_av, Lm.av.data(), sizeof(double) * Lm.av.size());
  std::memcpy(u_aj, Um.aj.data(), sizeof(int) * Um.aj.size());
  std::memcpy(u_av, Um.av.data(), sizeof(double) * Um.av.size());
  std::memcpy(d, D.data(), sizeof(double) * n);
  *lnnz = (int)Lm.aj.size();
  *unnz = (int)Um.aj.size();
}

// SplitTriangle<L|U> (matrix_utils.hpp:805-879): triangle incl. diagonal.
int la_ref_split_triangle(int uplo, int n, int base, const int *ai,
                          const int *aj, const double *av, int *t_ai,
                          int *t_aj, double *t_av) {
  CSRMatrixVec<int, int, double> T;
  if (uplo == 0)
    SplitTriangle<L>(n, base, ai, aj, av, T);
  else
    SplitTriangle<U>(n, base, ai, aj, av, T);
  std::memcpy(t_ai, T.ai.data(), sizeof(int) * (n + 1));
  std::memcpy(t_aj, T.aj.data(), sizeof(int) * T.aj.size());
  std::memcpy(t_av, T.av.data(), sizeof(double) * T.av.size());
  return (int)T.aj.size();
}

// ParallelTranspose2 (matrix_utils.hpp:311-390)
void la_ref_transpose(int rows, int cols, int base, const int *ai,
                      const int *aj, const double *av, int *t_ai, int *t_aj,
                      double *t_av) {
  ParallelTranspose2(rows, cols, base, ai, aj, av, t_ai, t_aj, t_av);
}

// permute (matrix_utils.hpp:429-472): B(i,:) = A(iperm[i],:), cols -> perm.
void la_ref_permute(int n, int base, const int *ai, const int *aj,
                    const double *av, const int *iperm, const int *perm,
                    int *p_ai, int *p_aj, double *p_av) {
  permute(n, base, ai, aj, av, iperm, perm, p_ai, p_aj, p_av);
}

// permuteVec (matrix_utils.hpp:562-576)
void la_ref_permute_vec(int n, int base, const double *v, const int *iperm, double *out) {
  permuteVec(n, base, v, iperm, out);
}

// inversePermute (utils/utils.cpp:101-108)
void la_ref_inverse_permute(int n, int base, const int *perm, int *iperm) {
  std::vector<MKL_INT> p(perm, perm + n), ip;
  utils::inversePermute(ip, p, base);
  std::memcpy(iperm, ip.data(), sizeof(int) * ip.size());
}

// Diagonal (matrix_utils.hpp:677-704); returns its bool
int la_ref_diagonal(int n, int base, const int *ai, const int *aj, const double *av,
                    int *diagpos, double *diag, int invert) {
  return Diagonal(n, base, ai, aj, av, diagpos, diag, invert != 0) ? 1 : 0;
}

// ValidCSR (matrix_utils.hpp:985-1014)
int la_ref_valid_csr(int rows, int cols, int base, const int *ai,
                     const int *aj) {
  return ValidCSR(rows, cols, base, ai, aj) ? 1 : 0;
}

// IC(0): ICCLevel0SymSymbolic + ICCLevelNumeric (precond.hpp:13-37, 615-693)
// on the upper triangle (diagonal first in each row) of an SPD matrix, with
// the diagonal position taken as the row start exactly as the reference's
// own test does (tests/precond_test.cpp:156-158).  Returns 1 on success and
// 0 on a negative pivot.
int la_ref_icc0(int n, int base, const int *u_ai, const int *u_aj,
                const double *u_av, double omega, double *icc_av) {
  CSRMatrixVec<int, int, double> icc;
  ICCLevel0SymSymbolic(n, base, u_ai, u_aj, icc);
  bool ok = ICCLevelNumeric(n, base, u_ai, u_aj, u_av, u_ai, 0, omega,
                            icc.ai.data(), icc.aj.data(), icc.av.data());
  std::memcpy(icc_av, icc.av.data(), sizeof(double) * icc.av.size());
  return ok ? 1 : 0;
}

// SerialCM, reverse Cuthill-McKee (reordering/Reordering.cpp:37-136)
void la_ref_serial_cm(int n, int base, const int *ai, const int *aj,
                      int *iperm, int *perm) {
  const int nnz = ai[n] - base;
  std::shared_ptr<int[]> sai(new int[n + 1]), saj(new int[nnz > 0 ? nnz : 1]);
  std::memcpy(sai.get(), ai, sizeof(int) * (n + 1));
  std::memcpy(saj.get(), aj, sizeof(int) * nnz);
  mkl_wrapper::mkl_sparse_mat m(n, n, sai, saj, base);
  std::vector<int> ip, p;
  reordering::SerialCM(&m, ip, p);
  std::memcpy(iperm, ip.data(), sizeof(int) * n);
  std::memcpy(perm, p.data(), sizeof(int) * n);
}

// ------------------------------------------------ CPU IC(0)-PCG baseline
// The reference's PCG driver (mkl_wrapper/mkl_solver.cpp:150-251) needs MKL,
// which is absent, so the CPU baseline PCG is COMPOSED FROM REFERENCE
// KERNELS: ParallelSPMV for A*p, OptimizedTriangularSolve<Barrier, L> on
// L = U^T (with diagonal) then <Barrier, U> (with diagonal) for the IC(0)
// apply, and OpenMP FP64 dots/axpys; the loop itself is this shim's.  It
// stops on the true residual ||b - A x|| / ||b|| < rtol, the reference's
// user stopping test (mkl_solver.cpp:211-225), checked when the recurrence
// residual drops below rtol.  x0 = 0.  Returns the iteration count
// (negative if maxit was reached).
struct RefPcg {
  int n, base, nthreads;
  const int *ai, *aj;
  const double *av;
  std::vector<int> lai, laj, uai, uaj;
  std::vector<double> lav, uav, diag;
  void *lsolve, *usolve;
};

void *la_ref_pcg_create(int nthreads, int n, int base, const int *ai,
                        const int *aj, const double *av, const int *u_ai,
                        const int *u_aj, const double *icc_av) {
  // icc factor U (upper, diagonal first, A ~= U^T U) -> strict U + diag,
  // and strict L = transpose(strict U) with the same diagonal.
  auto *p = new RefPcg{};
  p->n = n;
  p->base = base;
  p->nthreads = nthreads;
  p->ai = ai;
  p->aj = aj;
  p->av = av;
  omp_set_num_threads(nthreads);
  CSRMatrixVec<int, int, double> Ls, Us;
  std::vector<double> D;
  SplitLDU(n, base, u_ai, u_aj, icc_av, Ls, D, Us);
  p->diag = D;
  p->uai = Us.ai;
  p->uaj = Us.aj;
  p->uav = Us.av;
  const int unnz = (int)Us.aj.size();
  p->lai.resize(n + 1);
  p->laj.resize(unnz > 0 ? unnz : 1);
  p->lav.resize(unnz > 0 ? unnz : 1);
  ParallelTranspose2(n, n, base, p->uai.data(), p->uaj.data(), p->uav.data(),
                     p->lai.data(), p->laj.data(), p->lav.data());
  p->lsolve = la_ref_trsv_create(0, 0, nthreads, n, base, p->lai.data(),
                                 p->laj.data(), p->lav.data(), p->diag.data());
  p->usolve = la_ref_trsv_create(0, 1, nthreads, n, base, p->uai.data(),
                                 p->uaj.data(), p->uav.data(), p->diag.data());
  return p;
}

static double dot(int n, const double *a, const double *b) {
  double s = 0;
#pragma omp parallel for reduction(+ : s)
  for (int i = 0; i < n; i++)
    s += a[i] * b[i];
  return s;
}

int la_ref_pcg_solve(void *hv, const double *b, double *x, double rtol,
                     int maxit, double *final_rel_resid) {
  auto *p = static_cast<RefPcg *>(hv);
  const int n = p->n;
  omp_set_num_threads(p->nthreads);
  std::vector<double> r(n), z(n), q(n), pp(n), t(n);
  ParallelSPMV spmv;
#pragma omp parallel for
  for (int i = 0; i < n; i++) {
    x[i] = 0;
    r[i] = b[i];
  }
  const double bnorm = std::sqrt(dot(n, b, b));
  if (bnorm == 0) {
    *final_rel_resid = 0;
    return 0;
  }
  la_ref_trsv_apply(p->lsolve, r.data(), t.data());
  la_ref_trsv_apply(p->usolve, t.data(), z.data());
  std::copy(z.begin(), z.end(), pp.begin());
  double rz = dot(n, r.data(), z.data());
  int it = 0;
  double rel = 1.0;
  for (it = 1; it <= maxit; it++) {
    spmv(n, p->base, p->ai, p->aj, p->av, pp.data(), q.data(), 1.0, 0.0);
    const double alpha = rz / dot(n, pp.data(), q.data());
#pragma omp parallel for
    for (int i = 0; i < n; i++) {
      x[i] += alpha * pp[i];
      r[i] -= alpha * q[i];
    }
    const double rn = std::sqrt(dot(n, r.data(), r.data()));
    if (rn / bnorm < rtol) {
      spmv(n, p->base, p->ai, p->aj, p->av, x, t.data(), 1.0, 0.0);
#pragma omp parallel for
      for (int i = 0; i < n; i++)
        t[i] = b[i] - t[i];
      rel = std::sqrt(dot(n, t.data(), t.data())) / bnorm;
      if (rel < rtol) {
        *final_rel_resid = rel;
        return it;
      }
    }
    la_ref_trsv_apply(p->lsolve, r.data(), t.data());
    la_ref_trsv_apply(p->usolve, t.data(), z.data());
    const double rz_new = dot(n, r.data(), z.data());
    const double beta = rz_new / rz;
    rz = rz_new;
#pragma omp parallel for
    for (int i = 0; i < n; i++)
      pp[i] = z[i] + beta * pp[i];
  }
  spmv(n, p->base, p->ai, p->aj, p->av, x, t.data(), 1.0, 0.0);
  for (int i = 0; i < n; i++)
    t[i] = b[i] - t[i];
  *final_rel_resid = std::sqrt(dot(n, t.data(), t.data())) / bnorm;
  return -maxit;
}

void la_ref_pcg_destroy(void *hv) {
  auto *p = static_cast<RefPcg *>(hv);
  la_ref_trsv_destroy(p->lsolve);
  la_ref_trsv_destroy(p->usolve);
  delete p;
}

} // extern "C"
