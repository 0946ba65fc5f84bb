/* la_oracle.c -- TEST INFRASTRUCTURE ONLY: the CPU oracle.
 *
 * A plain-C, single-threaded restatement of the reference's algorithms on
 * the sparse hot path (miaodi/linearAlgebra).  It is the checker for the
 * CUDA product: only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg load it (as oracle/liboracle.so), never the product.
 *
 * Pinning: tests/test_oracle.py checks every function here against the
 * reference's own code compiled in place (oracle/_ref/libla_ref.so, built by
 * oracle/Makefile) and against the committed fixtures in tests/golden/.
 * The multi-threaded reference kernels are restated with an explicit chunk
 * count T standing for the reference's OpenMP thread count, so that with the
 * same T the oracle reproduces the reference's summation order exactly.
 *
 * Conventions follow the reference: int32 indices, double values, index
 * base 0 or 1 subtracted on every access, y = alpha * A * x + beta * y.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* utils/utils.h:176-185 LoadBalancedPartitionPos: even split of `total`
 * items over `parts`, the first (total % parts) parts one item larger. */
static void balanced_range(long total, int tid, int parts, long *s, long *e) {
  long w = total / parts, r = total % parts;
  if (tid >= r) {
    *s = tid * w + r;
    *e = (tid + 1) * w + r;
  } else {
    *s = tid * (w + 1);
    *e = (tid + 1) * (w + 1);
  }
}

/* ------------------------------------------------------------------ SpMV */

/* spmv.hpp:12-29 SerialSPMV: row-by-row, sequential in-row sum;
 * x[i] = alpha * sum + (beta == 0 ? 0 : beta * x[i]). */
void oracle_serial_spmv(int n, int base, const int *ai, const int *aj,
                        const double *av, const double *b, double *x,
                        double alpha, double beta) {
  for (int i = 0; i < n; i++) {
    double v = 0;
    for (int j = ai[i] - base; j < ai[i + 1] - base; j++)
      v += av[j] * b[aj[j] - base];
    x[i] = alpha * v + (beta == 0 ? 0 : beta * x[i]);
  }
}

/* spmv.hpp:59-185 SegSumSPMV with T chunks.  Phase 1 marks row heads,
 * phase 2 forms alpha*av*b per nonzero with an in-chunk segmented inclusive
 * scan (head flags propagated forward), phase 3 scans the T chunk carries
 * serially, phase 4 adds the carry to each chunk's leading open segment,
 * phase 5 writes x[i] = product[last nz of row i] + beta * x[i].
 * Unlike the reference (spmv.hpp:95 writes flag index nnz for trailing
 * empty rows, one past its buffer), the flag array here has nnz + 1 bytes. */
static void segsum_core(int T, const long *pre, int n, int base,
                        const int *ai, const int *aj, const double *av,
                        const double *b, double *x, double alpha,
                        double beta) {
  const long nnz = (long)ai[n] - base;
  unsigned char *bv = calloc((size_t)nnz + 1, 1);
  double *prod = malloc(sizeof(double) * (size_t)(nnz > 0 ? nnz : 1));
  unsigned char *tbv = calloc((size_t)T + 1, 1);
  double *tprod = calloc((size_t)T + 1, sizeof(double));
  for (int i = 0; i < n; i++)
    bv[ai[i] - base] = 1;
  for (int t = 0; t < T; t++) {
    const long s = pre[t], e = pre[t + 1];
    for (long i = s; i < e; i++) {
      prod[i] = alpha * av[i] * b[aj[i] - base];
      if (i > s && !bv[i]) {
        prod[i] += prod[i - 1];
        if (bv[i - 1])
          bv[i] = 1;
      }
    }
    tprod[t + 1] = 0;
    if (s < e) {
      tprod[t + 1] = prod[e - 1];
      if (bv[e - 1])
        tbv[t + 1] = 1;
    }
  }
  for (int i = 1; i <= T; i++) {
    if (!tbv[i]) {
      tprod[i] += tprod[i - 1];
      if (tbv[i - 1])
        tbv[i] = 1;
    }
  }
  for (int t = 0; t < T; t++) {
    const long s = pre[t], e = pre[t + 1];
    for (long i = s; i < e; i++) {
      if (bv[i])
        break;
      prod[i] += tprod[t];
    }
  }
  for (int i = 0; i < n; i++) {
    if (ai[i + 1] > ai[i])
      x[i] = prod[ai[i + 1] - base - 1] + beta * x[i];
    else
      x[i] = beta * x[i];
  }
  free(bv);
  free(prod);
  free(tbv);
  free(tprod);
}

/* Chunk prefixes: the reference's balanced split of nnz over T workers
 * (utils.h:176-185, spmv.hpp:99 and :202-208), or fixed chunks of `tile`
 * nonzeros (the GPU tiles), T = ceil(nnz / tile). */
static long *balanced_prefix(long nnz, int T) {
  long *pre = malloc(sizeof(long) * ((size_t)T + 1));
  for (int t = 0; t < T; t++) {
    long s, e;
    balanced_range(nnz, t, T, &s, &e);
    pre[t] = s;
    pre[t + 1] = e;
  }
  return pre;
}
static long *tiled_prefix(long nnz, int tile, int *T) {
  *T = nnz == 0 ? 1 : (int)((nnz + tile - 1) / tile);
  long *pre = malloc(sizeof(long) * ((size_t)*T + 1));
  for (int t = 0; t <= *T; t++)
    pre[t] = (long)t * tile < nnz ? (long)t * tile : nnz;
  return pre;
}

void oracle_segsum_spmv(int T, int n, int base, const int *ai, const int *aj,
                        const double *av, const double *b, double *x,
                        double alpha, double beta) {
  long *pre = balanced_prefix((long)ai[n] - base, T);
  segsum_core(T, pre, n, base, ai, aj, av, b, x, alpha, beta);
  free(pre);
}

/* SegSumSPMV's algorithm over fixed chunks of `tile` nonzeros. */
void oracle_segsum_spmv_tiled(int tile, int n, int base, const int *ai,
                              const int *aj, const double *av, const double *b,
                              double *x, double alpha, double beta) {
  int T;
  long *pre = tiled_prefix((long)ai[n] - base, tile, &T);
  segsum_core(T, pre, n, base, ai, aj, av, b, x, alpha, beta);
  free(pre);
}

/* First index p in ai[0..n] with ai[p] > v (std::upper_bound). */
static int upper_bound_int(const int *a, int len, long v) {
  int lo = 0, hi = len;
  while (lo < hi) {
    int mid = lo + (hi - lo) / 2;
    if (a[mid] > v)
      hi = mid;
    else
      lo = mid + 1;
  }
  return lo;
}

/* spmv.hpp:186-300 ALBUSSPMV with T blocks.  preprocess (:195-228): the
 * nnz are split into T equal blocks, block t starting in row
 * upper_bound(ai, prefix[t] + base) - 1.  apply (:230-293): each block
 * sums its partial first row into boundary[2t], writes whole interior rows
 * directly, sums its partial last row into boundary[2t+1]; then a serial
 * merge scales each boundary row by beta once and adds the partials in
 * block order.  The reference leaves rows that precede the first block's
 * start row untouched (leading empty rows); this restatement does the same. */
static void albus_core(int T, const long *pre, int n, int base,
                       const int *ai, const int *aj, const double *av,
                       const double *b, double *x, double alpha, double beta) {
  int *srow = malloc(sizeof(int) * ((size_t)T + 1));
  double *bnd = calloc(2 * (size_t)T, sizeof(double));
  for (int i = 0; i <= T; i++)
    srow[i] = upper_bound_int(ai, n + 1, pre[i] + base) - 1;
  for (int t = 0; t < T; t++) {
    int start = srow[t], end = srow[t + 1];
    double v;
    if (start < end) {
      v = 0;
      for (long j = pre[t]; j < ai[start + 1] - base; j++)
        v += av[j] * b[aj[j] - base];
      start++;
      bnd[2 * t] = alpha * v;
      for (int i = start; i < end; i++) {
        v = 0;
        for (long j = ai[i] - base; j < ai[i + 1] - base; j++)
          v += av[j] * b[aj[j] - base];
        x[i] = alpha * v + (beta == 0 ? 0 : beta * x[i]);
      }
      v = 0;
      for (long j = ai[end] - base; j < pre[t + 1]; j++)
        v += av[j] * b[aj[j] - base];
      bnd[2 * t + 1] = alpha * v;
    } else {
      v = 0;
      for (long j = pre[t]; j < pre[t + 1]; j++)
        v += av[j] * b[aj[j] - base];
      bnd[2 * t] = alpha * v;
      bnd[2 * t + 1] = 0;
    }
  }
  /* With more chunks than nonzeros the trailing empty chunks start at row n
   * and the reference's merge writes x[n], one past the output
   * (spmv.hpp:275-292); rows >= n are skipped here (their partials are 0). */
  int idx = -1;
  for (int t = 0; t < T; t++) {
    if (srow[t] != idx) {
      idx = srow[t];
      if (idx < n)
        x[idx] *= beta;
    }
    if (idx < n)
      x[idx] += bnd[2 * t];
    if (t == T - 1)
      break;
    if (srow[t + 1] != idx) {
      idx = srow[t + 1];
      if (idx < n)
        x[idx] *= beta;
    }
    if (idx < n)
      x[idx] += bnd[2 * t + 1];
  }
  free(srow);
  free(bnd);
}

void oracle_albus_spmv(int T, int n, int base, const int *ai, const int *aj,
                       const double *av, const double *b, double *x,
                       double alpha, double beta) {
  long *pre = balanced_prefix((long)ai[n] - base, T);
  albus_core(T, pre, n, base, ai, aj, av, b, x, alpha, beta);
  free(pre);
}

/* ALBUSSPMV's algorithm over fixed chunks of `tile` nonzeros. */
void oracle_albus_spmv_tiled(int tile, int n, int base, const int *ai,
                             const int *aj, const double *av, const double *b,
                             double *x, double alpha, double beta) {
  int T;
  long *pre = tiled_prefix((long)ai[n] - base, tile, &T);
  albus_core(T, pre, n, base, ai, aj, av, b, x, alpha, beta);
  free(pre);
}

/* Transposed product y = alpha * A^T g + beta * y, the SpMV adjoint
 * (dL/dx for y = A x).  Column scatter in row order, as ForwardSubstitutionT
 * (triangle_solve.hpp:87-98) scatters. */
void oracle_spmv_transpose(int n, int ncols, int base, const int *ai,
                           const int *aj, const double *av, const double *g,
                           double *y, double alpha, double beta) {
  for (int c = 0; c < ncols; c++)
    y[c] = beta == 0 ? 0 : beta * y[c];
  for (int i = 0; i < n; i++)
    for (int j = ai[i] - base; j < ai[i + 1] - base; j++)
      y[aj[j] - base] += alpha * av[j] * g[i];
}

/* Sampled outer product over the pattern: d[k] = alpha * g[row(k)] *
 * x[col(k)], the SpMV adjoint with respect to the stored values. */
void oracle_sddmm_pattern(int n, int base, const int *ai, const int *aj,
                          const double *g, const double *x, double *d,
                          double alpha) {
  for (int i = 0; i < n; i++)
    for (int j = ai[i] - base; j < ai[i + 1] - base; j++)
      d[j] = alpha * g[i] * x[aj[j] - base];
}

/* ----------------------------------------------------- triangular solves */

/* triangle_solve.hpp:32-43: strict-lower L, unit diagonal. */
void oracle_forward_substitution(int n, int base, const int *ai, const int *aj,
                                 const double *av, const double *b, double *x) {
  for (int i = 0; i < n; i++) {
    double v = 0;
    for (int j = ai[i] - base; j < ai[i + 1] - base; j++)
      v += av[j] * x[aj[j] - base];
    x[i] = b[i] - v;
  }
}

/* Non-unit lower solve: x_i = (b_i - sum_j L_ij x_j) / diag_i, the form
 * OptimizedTriangularSolve<.., L> takes with a diagonal
 * (triangle_solve.tpp:147). */
void oracle_forward_substitution_diag(int n, int base, const int *ai,
                                      const int *aj, const double *av,
                                      const double *diag, const double *b,
                                      double *x) {
  for (int i = 0; i < n; i++) {
    double v = 0;
    for (int j = ai[i] - base; j < ai[i + 1] - base; j++)
      v += av[j] * x[aj[j] - base];
    x[i] = diag ? (b[i] - v) / diag[i] : b[i] - v;
  }
}

/* triangle_solve.hpp:59-71: strict-upper U with diagonal. A null diag is
 * the unit-diagonal form. */
void oracle_backward_substitution(int n, int base, const int *ai,
                                  const int *aj, const double *av,
                                  const double *diag, const double *b,
                                  double *x) {
  for (int i = n - 1; i >= 0; i--) {
    double v = 0;
    for (int j = ai[i] - base; j < ai[i + 1] - base; j++)
      v += av[j] * x[aj[j] - base];
    x[i] = diag ? (b[i] - v) / diag[i] : b[i] - v;
  }
}

/* triangle_solve.hpp:87-98: solve with L = U^T given the CSR of strict U,
 * unit diagonal, by column scatter. */
void oracle_forward_substitution_t(int n, int base, const int *ai,
                                   const int *aj, const double *av,
                                   const double *b, double *x) {
  memcpy(x, b, sizeof(double) * (size_t)n);
  for (int i = 0; i < n; i++)
    for (int j = ai[i] - base; j < ai[i + 1] - base; j++)
      x[aj[j] - base] -= av[j] * x[i];
}

/* triangle_solve.hpp:100-145 level-scheduled apply, levels visited in
 * order, rows of a level in iperm order. */
void oracle_level_solve(int nlev, const int *iperm, const int *prefix,
                        int base, const int *ai, const int *aj,
                        const double *av, const double *diag, const double *b,
                        double *x) {
  for (int l = 0; l < nlev; l++)
    for (int p = prefix[l]; p < prefix[l + 1]; p++) {
      int i = iperm[p] - base;
      double v = 0;
      for (int j = ai[i] - base; j < ai[i + 1] - base; j++)
        v += av[j] * x[aj[j] - base];
      x[i] = diag ? (b[i] - v) / diag[i] : b[i] - v;
    }
}

/* The same level-scheduled apply with FP32 storage and FP32 arithmetic: the
 * factor values and the diagonal rounded to float once (as the FP32 plans
 * store them), every product, sum, difference and quotient a single float
 * operation (ISO C: no contraction into FMAs, FLT_EVAL_METHOD 0 on x86-64),
 * so an FP32 solve in the reference's row order is reproduced bit for bit. */
void oracle_level_solve_f32(int nlev, const int *iperm, const int *prefix,
                            int base, const int *ai, const int *aj,
                            const double *av, const double *diag, const float *b,
                            float *x) {
  for (int l = 0; l < nlev; l++)
    for (int p = prefix[l]; p < prefix[l + 1]; p++) {
      int i = iperm[p] - base;
      float v = 0.0f;
      for (int j = ai[i] - base; j < ai[i + 1] - base; j++) {
        const float prod = (float)av[j] * x[aj[j] - base];
        v = v + prod;
      }
      const float r = b[i] - v;
      x[i] = diag ? r / (float)diag[i] : r;
    }
}

/* ------------------------------------------------------- level scheduling */

/* matrix_utils.hpp:637-675 TopologicalSort2<L|U> (uplo 0 / 1): depth of
 * row i = max over its entries j of depth[j] + 1 (rows visited ascending for
 * L, descending for U), levels = max depth + 1, then a counting sort gives
 * iperm ordered by (level, row ascending) with iperm values i + base and a
 * zero-based prefix[levels + 1].  Returns the level count. */
int oracle_topological_sort2(int uplo, int n, int base, const int *ai,
                             const int *aj, int *iperm, int *prefix) {
  int *deg = calloc((size_t)n + 1, sizeof(int));
  int levels = 0;
  for (int k = 0; k < n; k++) {
    int i = uplo == 0 ? k : n - 1 - k;
    for (int j = ai[i] - base; j < ai[i + 1] - base; j++) {
      int d = deg[aj[j] - base] + 1;
      if (d > deg[i])
        deg[i] = d;
    }
    if (deg[i] + 1 > levels)
      levels = deg[i] + 1;
  }
  for (int l = 0; l <= levels; l++)
    prefix[l] = 0;
  for (int i = 0; i < n; i++)
    prefix[deg[i] + 1]++;
  for (int l = 0; l < levels; l++)
    prefix[l + 1] += prefix[l];
  /* prefix[l] now holds the start of level l; place rows ascending. */
  int *pos = malloc(sizeof(int) * ((size_t)levels + 1));
  memcpy(pos, prefix, sizeof(int) * ((size_t)levels + 1));
  for (int i = 0; i < n; i++)
    iperm[pos[deg[i]]++] = i + base;
  free(pos);
  free(deg);
  return levels;
}

/* ------------------------------------------------------ matrix utilities */

/* matrix_utils.hpp:720-803 SplitLDU: strict L, diagonal D (0 if absent),
 * strict U, column order kept.  Outputs sized by the caller (nnz, n + 1). */
void oracle_split_ldu(int n, int base, const int *ai, const int *aj,
                      const double *av, int *l_ai, int *l_aj, double *l_av,
                      double *d, int *u_ai, int *u_aj, double *u_av, int *lnnz,
                      int *unnz) {
  int lp = 0, up = 0;
  l_ai[0] = base;
  u_ai[0] = base;
  for (int i = 0; i < n; i++) {
    d[i] = 0;
    for (int j = ai[i] - base; j < ai[i + 1] - base; j++) {
      int c = aj[j] - base;
      if (c < i) {
        l_aj[lp] = aj[j];
        l_av[lp++] = av[j];
      } else if (c == i) {
        d[i] = av[j];
      } else {
        u_aj[up] = aj[j];
        u_av[up++] = av[j];
      }
    }
    l_ai[i + 1] = lp + base;
    u_ai[i + 1] = up + base;
  }
  *lnnz = lp;
  *unnz = up;
}

/* matrix_utils.hpp:805-879 SplitTriangle<L|U>: the triangle including the
 * diagonal.  Returns its nnz. */
int oracle_split_triangle(int uplo, int n, int base, const int *ai,
                          const int *aj, const double *av, int *t_ai,
                          int *t_aj, double *t_av) {
  int p = 0;
  t_ai[0] = base;
  for (int i = 0; i < n; i++) {
    for (int j = ai[i] - base; j < ai[i + 1] - base; j++) {
      int c = aj[j] - base;
      if ((uplo == 1 && c >= i) || (uplo == 0 && c <= i)) {
        t_aj[p] = aj[j];
        t_av[p++] = av[j];
      }
    }
    t_ai[i + 1] = p + base;
  }
  return p;
}

/* matrix_utils.hpp:195-225 SerialTranspose (ParallelTranspose2 produces the
 * same arrays): rows of A^T list source rows ascending. */
void oracle_transpose(int rows, int cols, int base, const int *ai,
                      const int *aj, const double *av, int *t_ai, int *t_aj,
                      double *t_av) {
  int *cnt = calloc((size_t)cols + 1, sizeof(int));
  for (int j = 0; j < ai[rows] - base; j++)
    cnt[aj[j] - base + 1]++;
  for (int c = 0; c < cols; c++)
    cnt[c + 1] += cnt[c];
  for (int c = 0; c <= cols; c++)
    t_ai[c] = cnt[c] + base;
  for (int i = 0; i < rows; i++)
    for (int j = ai[i] - base; j < ai[i + 1] - base; j++) {
      int q = cnt[aj[j] - base]++;
      t_aj[q] = i + base;
      if (av && t_av)
        t_av[q] = av[j];
    }
  free(cnt);
}

/* ----------------------------------------------------------------- IC(0) */

/* precond.hpp:615-693 ICCLevelNumeric on the IC(0) pattern (= the upper
 * triangle of A, diagonal first in each row, precond.hpp:13-37).  Up-looking
 * row-by-row factorisation: row j starts as A's row j with the diagonal
 * multiplied by (1 + omega); every earlier row k with a stored entry in
 * column j (found through the same LIFO linked lists `llist` / cursor `jk`
 * the reference keeps) subtracts U_kj * U_k,: over the matching pattern;
 * then the pivot p is checked (p < 0 -> return 0, a breakdown), the row is
 * scaled U_jj = sqrt(p), U_ji = a_ji / sqrt(p).  A ~= U^T U.  u_* is the
 * upper triangle of A incl. diagonal; icc_av shares its pattern. */
int oracle_icc0(int n, int base, const int *u_ai, const int *u_aj,
                const double *u_av, double omega, double *icc_av) {
  const int NONE = 0x7fffffff;
  int *llist = malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  int *jk = malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  for (int i = 0; i < n; i++)
    llist[i] = NONE;
  for (int j = 0; j < n; j++) {
    const int rs = u_ai[j] - base, re = u_ai[j + 1] - base;
    icc_av[rs] = u_av[rs] * (1.0 + omega);
    for (int p = rs + 1; p < re; p++)
      icc_av[p] = u_av[p];
    int k = llist[j];
    while (k < j) {
      int ik = jk[k]++;
      const int ke = u_ai[k + 1] - base;
      int knext = llist[k];
      if (ik + 1 < ke) {
        int c = u_aj[ik + 1] - base;
        llist[k] = llist[c];
        llist[c] = k;
      }
      k = knext;
      const double ajk = icc_av[ik];
      int p = rs;
      while (ik < ke && p < re) {
        if (u_aj[ik] == u_aj[p])
          icc_av[p++] -= ajk * icc_av[ik++];
        else if (u_aj[ik] < u_aj[p])
          ik++;
        else
          p++;
      }
    }
    if (re - rs > 1) {
      int c = u_aj[rs + 1] - base;
      llist[j] = llist[c];
      llist[c] = j;
      jk[j] = rs + 1;
    }
    if (icc_av[rs] < 0) {
      free(llist);
      free(jk);
      return 0;
    }
    const double d = sqrt(icc_av[rs]);
    icc_av[rs] = d;
    for (int p = rs + 1; p < re; p++)
      icc_av[p] /= d;
  }
  free(llist);
  free(jk);
  return 1;
}

/* ------------------------------------------------------- RCM reordering */

/* reordering/Reordering.cpp:37-136 SerialCM, with the pieces it uses:
 * components (reordering/UnionFind.cpp:83-129, 217-293: ordered by their
 * largest node index, members ascending), the pseudo-peripheral source
 * (reordering/Reordering.h:72-136) and the CM sweep.
 *
 * PseudoDiameter, as the reference executes it: start from the component's
 * first minimum-degree node; BFS from it (height = level count); pick up to
 * five candidates from its last level greedily by (degree, index) and mark
 * each candidate and its neighbours with degree INT_MAX -- this mutation of
 * `degrees` persists and later breaks CM ties; BFS from the first candidate:
 * if it is deeper, it becomes the new source and the search repeats,
 * otherwise it is the target and the search ends.  (The reference's width
 * bookkeeping accumulates across one BFS object, so candidates after the
 * first can never win and the final source/target swap never fires; the
 * result is the rule stated here.)
 *
 * CM sweep: BFS levels from the source; visiting the ordering level by
 * level, each node appends its unvisited next-level neighbours sorted by
 * (mutated degree, index).  Finally the whole iperm is reversed and
 * perm = inverse(iperm).  Values carry the index base. */

/* BFS levels of the component containing src (zero-based); returns the
 * number of levels, fills lev (-1 = unreached) and the last level's nodes. */
static int bfs_levels(int n, int base, const int *ai, const int *aj, int src,
                      int *lev, int *queue, int *last, int *nlast) {
  for (int i = 0; i < n; i++)
    lev[i] = -1;
  int head = 0, tail = 0;
  queue[tail++] = src;
  lev[src] = 0;
  while (head < tail) {
    int u = queue[head++];
    for (int j = ai[u] - base; j < ai[u + 1] - base; j++) {
      int v = aj[j] - base;
      if (lev[v] == -1) {
        lev[v] = lev[u] + 1;
        queue[tail++] = v;
      }
    }
  }
  int h = lev[queue[tail - 1]] + 1;
  int c = 0;
  for (int q = 0; q < tail; q++)
    if (lev[queue[q]] == h - 1)
      last[c++] = queue[q];
  *nlast = c;
  return h;
}

static const int *g_sort_deg;
static int cmp_deg_idx(const void *a, const void *b) {
  int x = *(const int *)a, y = *(const int *)b;
  if (g_sort_deg[x] != g_sort_deg[y])
    return g_sort_deg[x] < g_sort_deg[y] ? -1 : 1;
  return x < y ? -1 : (x > y);
}

void oracle_rcm(int n, int base, const int *ai, const int *aj, int *iperm,
                int *perm) {
  const int INF = 0x7fffffff;
  int *deg = malloc(sizeof(int) * (size_t)n);
  int *comp = malloc(sizeof(int) * (size_t)n);
  int *lev = malloc(sizeof(int) * (size_t)n);
  int *queue = malloc(sizeof(int) * (size_t)n);
  int *last = malloc(sizeof(int) * (size_t)n);
  int *order = malloc(sizeof(int) * (size_t)n);
  int *cmax = malloc(sizeof(int) * (size_t)n);
  for (int i = 0; i < n; i++) {
    deg[i] = ai[i + 1] - ai[i];
    comp[i] = -1;
  }
  /* Components by BFS; label = discovery id, then ordered by max node. */
  int ncomp = 0;
  for (int i = 0; i < n; i++) {
    if (comp[i] != -1)
      continue;
    int head = 0, tail = 0, mx = i;
    queue[tail++] = i;
    comp[i] = ncomp;
    while (head < tail) {
      int u = queue[head++];
      if (u > mx)
        mx = u;
      for (int j = ai[u] - base; j < ai[u + 1] - base; j++) {
        int v = aj[j] - base;
        if (comp[v] == -1) {
          comp[v] = ncomp;
          queue[tail++] = v;
        }
      }
    }
    cmax[ncomp++] = mx;
  }
  /* Order components by their maximum node (a node is its component's
   * maximum exactly once; scanning ascending lists components in that
   * order), members ascending. */
  int *crank = malloc(sizeof(int) * (size_t)(ncomp > 0 ? ncomp : 1));
  int *cstart = calloc((size_t)ncomp + 1, sizeof(int));
  {
    int r = 0;
    for (int i = 0; i < n; i++)
      if (cmax[comp[i]] == i)
        crank[comp[i]] = r++;
    for (int i = 0; i < n; i++)
      cstart[crank[comp[i]] + 1]++;
    for (int c = 0; c < ncomp; c++)
      cstart[c + 1] += cstart[c];
    int *fill = malloc(sizeof(int) * (size_t)(ncomp > 0 ? ncomp : 1));
    memcpy(fill, cstart, sizeof(int) * (size_t)ncomp);
    for (int i = 0; i < n; i++)
      order[fill[crank[comp[i]]]++] = i;
    free(fill);
  }
  for (int c = 0; c < ncomp; c++) {
    const int off = cstart[c], sz = cstart[c + 1] - cstart[c];
    if (sz <= 2) {
      for (int q = 0; q < sz; q++)
        iperm[off + q] = order[off + q] + base;
      continue;
    }
    /* pseudo-peripheral source */
    int src = -1, best = INF;
    for (int q = off; q < off + sz; q++)
      if (deg[order[q]] < best) {
        best = deg[order[q]];
        src = order[q];
      }
    for (;;) {
      int nlast;
      int height = bfs_levels(n, base, ai, aj, src, lev, queue, last, &nlast);
      int first = -1, chosen = 0;
      while (chosen < 5) {
        int md = INF, sel = -1;
        for (int q = 0; q < nlast; q++) {
          int v = last[q];
          if (deg[v] < md) {
            md = deg[v];
            sel = v;
          } else if (deg[v] == md && v < sel) {
            sel = v;
          }
        }
        if (md == INF)
          break;
        if (first < 0)
          first = sel;
        chosen++;
        deg[sel] = INF;
        for (int j = ai[sel] - base; j < ai[sel + 1] - base; j++)
          deg[aj[j] - base] = INF;
      }
      if (first < 0)
        break; /* the reference would loop forever here */
      int nl2;
      int h2 = bfs_levels(n, base, ai, aj, first, lev, queue, last, &nl2);
      if (height < h2) {
        src = first;
        continue;
      }
      break;
    }
    /* CM sweep from src */
    int nlast;
    int height = bfs_levels(n, base, ai, aj, src, lev, queue, last, &nlast);
    int *lstart = calloc((size_t)height + 1, sizeof(int));
    for (int q = off; q < off + sz; q++)
      lstart[lev[order[q]] + 1]++;
    for (int l = 0; l < height; l++)
      lstart[l + 1] += lstart[l];
    int e = off;
    iperm[e++] = src + base;
    g_sort_deg = deg;
    for (int l = 0; l < height; l++) {
      for (int r = lstart[l]; r != lstart[l + 1]; r++) {
        int u = iperm[r + off] - base;
        int nch = 0;
        for (int j = ai[u] - base; j < ai[u + 1] - base; j++) {
          int v = aj[j] - base;
          if (lev[v] == l + 1) {
            last[nch++] = v;
            lev[v] = -1;
          }
        }
        qsort(last, (size_t)nch, sizeof(int), cmp_deg_idx);
        for (int q = 0; q < nch; q++)
          iperm[e++] = last[q] + base;
      }
    }
    free(lstart);
  }
  for (int i = 0; i < n / 2; i++) {
    int t = iperm[i];
    iperm[i] = iperm[n - 1 - i];
    iperm[n - 1 - i] = t;
  }
  for (int i = 0; i < n; i++)
    perm[iperm[i] - base] = i + base;
  free(deg);
  free(comp);
  free(lev);
  free(queue);
  free(last);
  free(order);
  free(cmax);
  free(crank);
  free(cstart);
}

/* matrix_utils.hpp:429-472 permute: B(i,:) = A(iperm[i],:) with columns
 * mapped through perm and each row re-sorted by column. */
void oracle_permute(int n, int base, const int *ai, const int *aj,
                    const double *av, const int *iperm, const int *perm,
                    int *p_ai, int *p_aj, double *p_av) {
  p_ai[0] = base;
  for (int i = 0; i < n; i++) {
    int src = iperm[i] - base;
    p_ai[i + 1] = p_ai[i] + (ai[src + 1] - ai[src]);
  }
  for (int i = 0; i < n; i++) {
    int src = iperm[i] - base;
    int o = p_ai[i] - base, len = ai[src + 1] - ai[src];
    for (int q = 0; q < len; q++) {
      int c = aj[ai[src] - base + q];
      p_aj[o + q] = perm ? perm[c - base] : c;
      p_av[o + q] = av[ai[src] - base + q];
    }
    for (int a = 1; a < len; a++) { /* stable insertion sort by column */
      int kc = p_aj[o + a];
      double kv = p_av[o + a];
      int b = a - 1;
      while (b >= 0 && p_aj[o + b] > kc) {
        p_aj[o + b + 1] = p_aj[o + b];
        p_av[o + b + 1] = p_av[o + b];
        b--;
      }
      p_aj[o + b + 1] = kc;
      p_av[o + b + 1] = kv;
    }
  }
}

/* ------------------------------------------------------------- IC(0)-PCG */

/* IC(0)-preconditioned CG in FP64, x0 = 0, the reference's intended
 * sequence (execs/linearSolve.cpp:118-135, mkl_wrapper/mkl_solver.cpp:
 * 150-251): z = U^-1 U^-T r through the factor apply of
 * mkl_wrapper/incomplete_cholesky.cpp:21-29; stop when the true residual
 * ||b - A x|| / ||b|| < rtol (mkl_solver.cpp:211-225), checked once the
 * recurrence residual is below rtol.  u_* / icc_av: the IC(0) factor U
 * (upper, diagonal first).  Returns iterations, negative if maxit hit. */
static double odot(int n, const double *a, const double *b) {
  double s = 0;
  for (int i = 0; i < n; i++)
    s += a[i] * b[i];
  return s;
}

static void icc_apply(int n, int base, const int *u_ai, const int *u_aj,
                      const double *icc_av, const double *r, double *t,
                      double *z) {
  /* U^T t = r: forward, column-oriented over the rows of U */
  memcpy(t, r, sizeof(double) * (size_t)n);
  for (int i = 0; i < n; i++) {
    const int rs = u_ai[i] - base, re = u_ai[i + 1] - base;
    t[i] /= icc_av[rs];
    for (int j = rs + 1; j < re; j++)
      t[u_aj[j] - base] -= icc_av[j] * t[i];
  }
  /* U z = t: backward */
  for (int i = n - 1; i >= 0; i--) {
    const int rs = u_ai[i] - base, re = u_ai[i + 1] - base;
    double v = 0;
    for (int j = rs + 1; j < re; j++)
      v += icc_av[j] * z[u_aj[j] - base];
    z[i] = (t[i] - v) / icc_av[rs];
  }
}

int oracle_pcg(int n, int base, const int *ai, const int *aj, const double *av,
               const int *u_ai, const int *u_aj, const double *icc_av,
               const double *b, double *x, double rtol, int maxit,
               double *final_rel) {
  double *r = malloc(sizeof(double) * (size_t)n);
  double *z = malloc(sizeof(double) * (size_t)n);
  double *p = malloc(sizeof(double) * (size_t)n);
  double *q = malloc(sizeof(double) * (size_t)n);
  double *t = malloc(sizeof(double) * (size_t)n);
  int it, ret = -maxit;
  for (int i = 0; i < n; i++) {
    x[i] = 0;
    r[i] = b[i];
  }
  const double bn = sqrt(odot(n, b, b));
  *final_rel = 0;
  if (bn == 0) {
    ret = 0;
    goto done;
  }
  icc_apply(n, base, u_ai, u_aj, icc_av, r, t, z);
  memcpy(p, z, sizeof(double) * (size_t)n);
  double rz = odot(n, r, z);
  for (it = 1; it <= maxit; it++) {
    oracle_serial_spmv(n, base, ai, aj, av, p, q, 1.0, 0.0);
    const double alpha = rz / odot(n, p, q);
    for (int i = 0; i < n; i++) {
      x[i] += alpha * p[i];
      r[i] -= alpha * q[i];
    }
    if (sqrt(odot(n, r, r)) / bn < rtol) {
      oracle_serial_spmv(n, base, ai, aj, av, x, t, 1.0, 0.0);
      for (int i = 0; i < n; i++)
        t[i] = b[i] - t[i];
      double rel = sqrt(odot(n, t, t)) / bn;
      if (rel < rtol) {
        *final_rel = rel;
        ret = it;
        goto done;
      }
    }
    icc_apply(n, base, u_ai, u_aj, icc_av, r, t, z);
    const double rzn = odot(n, r, z);
    const double beta = rzn / rz;
    rz = rzn;
    for (int i = 0; i < n; i++)
      p[i] = z[i] + beta * p[i];
  }
  oracle_serial_spmv(n, base, ai, aj, av, x, t, 1.0, 0.0);
  for (int i = 0; i < n; i++)
    t[i] = b[i] - t[i];
  *final_rel = sqrt(odot(n, t, t)) / bn;
done:
  free(r);
  free(z);
  free(p);
  free(q);
  free(t);
  return ret;
}
