// la_host.cpp -- host-side preprocessing of the sparse hot path.
//
// These run once per matrix on the host, as in the reference, and their
// integer outputs (level sets, permutations, split patterns) must be
// bit-identical to the reference's; floating-point outputs (IC(0) values)
// follow the reference's operation order so they are bit-identical too.
// Each function cites the reference routine it restates.

#include "la_internal.h"

#include <omp.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <memory>
#include <numeric>

namespace la {

// matrix_utils.hpp:985-1014 ValidCSR.
bool valid_csr(int rows, int cols, int base, const int *ai, const int *aj,
               std::string *why) {
  auto fail = [&](const char *m, long r) {
    if (why) {
      char buf[128];
      std::snprintf(buf, sizeof buf, "%s (row %ld)", m, r);
      *why = buf;
    }
    return false;
  };
  if (rows < 0 || cols < 0)
    return fail("negative dimension", -1);
  if (ai[0] != base)
    return fail("ai[0] is not equal to base", 0);
  for (int i = 0; i < rows; i++) {
    if (ai[i + 1] < ai[i])
      return fail("ai is not monotonically increasing", i);
    const int *b = aj + (ai[i] - base), *e = aj + (ai[i + 1] - base);
    for (const int *p = b; p + 1 < e; p++) {
      if (p[1] < p[0])
        return fail("unsorted row", i);
      if (p[1] == p[0])
        return fail("duplicate entry in row", i);
    }
    if (e > b && (b[0] < base || e[-1] >= cols + base))
      return fail("column index out of range in row", i);
  }
  return true;
}

// matrix_utils.hpp:583-635 TopologicalSort (Kahn's breadth-first order):
// the same level sets as TopologicalSort2, another order inside a level.
// Level 0 holds the rows without entries, ascending (L) or descending (U);
// each later level lists, for the rows of the level before in their order,
// the rows that read them (ascending, the order of a stable transpose) as
// the last of their entries is consumed.  Returns the reference's value: the
// index of the last level (levels - 1, 0 for n == 0); prefix gets that + 2
// entries.  -1 when a level adds no row before all are placed (a cycle: not
// a triangle), where the reference would not stop.
int topological_sort_kahn(int uplo, int n, int base, const int *ai, const int *aj, int *iperm,
                          int *prefix) {
  std::vector<int> pending(n);
  int placed = 0, np = 2;
  prefix[0] = 0;
  prefix[1] = 0;
  for (int t = 0; t < n; t++) {
    const int i = uplo == 0 ? t : n - 1 - t;
    pending[i] = ai[i + 1] - ai[i];
    if (pending[i] == 0) {
      iperm[placed++] = i + base;
      prefix[1]++;
    }
  }
  // readers of each row, ascending
  const int nnz = ai[n] - base;
  std::vector<int> r_ptr(n + 1, 0), r_row(std::max(nnz, 1));
  for (int k = 0; k < nnz; k++)
    r_ptr[aj[k] - base + 1]++;
  for (int i = 0; i < n; i++)
    r_ptr[i + 1] += r_ptr[i];
  {
    std::vector<int> fill(r_ptr.begin(), r_ptr.end() - 1);
    for (int i = 0; i < n; i++)
      for (int k = ai[i] - base; k < ai[i + 1] - base; k++)
        r_row[fill[aj[k] - base]++] = i;
  }
  int level = 0;
  while (placed != n) {
    prefix[np] = prefix[np - 1];
    np++;
    for (int p = prefix[level]; p < prefix[level + 1]; p++) {
      const int row = iperm[p] - base;
      for (int k = r_ptr[row]; k < r_ptr[row + 1]; k++)
        if (--pending[r_row[k]] == 0) {
          iperm[placed++] = r_row[k] + base;
          prefix[np - 1]++;
        }
    }
    if (prefix[np - 1] == prefix[np - 2])
      return -1;
    level++;
  }
  return level;
}

// matrix_utils.hpp:637-675 TopologicalSort2.  depth(i) = max over stored
// entries j of depth(j) + 1, rows visited ascending (L) or descending (U);
// iperm lists rows by (level, ascending row) with values i + base; prefix is
// zero-based with levels + 1 entries.
int topological_sort2(int uplo, int n, int base, const int *ai, const int *aj,
                      int *iperm, int *prefix) {
  std::vector<int> depth(n, 0);
  int levels = 0;
  for (int k = 0; k < n; k++) {
    const int i = uplo == LA_LOWER ? k : n - 1 - k;
    int d = depth[i];
    for (int j = ai[i] - base; j < ai[i + 1] - base; j++)
      d = std::max(d, depth[aj[j] - base] + 1);
    depth[i] = d;
    levels = std::max(levels, d + 1);
  }
  std::fill(prefix, prefix + levels + 1, 0);
  for (int i = 0; i < n; i++)
    prefix[depth[i] + 1]++;
  for (int l = 0; l < levels; l++)
    prefix[l + 1] += prefix[l];
  std::vector<int> cursor(prefix, prefix + levels);
  for (int i = 0; i < n; i++)
    iperm[cursor[depth[i]]++] = i + base;
  return levels;
}

// matrix_utils.hpp:311-390 ParallelTranspose2 (same arrays as the serial
// form :195-225): a counting sort by column, stable in the source row.
void transpose(int rows, int cols, int base, const int *ai, const int *aj,
               const double *av, int *t_ai, int *t_aj, double *t_av) {
  const int nnz = ai[rows] - base;
  const bool vals = av && t_av;
  if (nnz < (1 << 18)) { // small: one pass in row order
    std::vector<int> pos(cols + 1, 0);
    for (int k = 0; k < nnz; k++)
      pos[aj[k] - base + 1]++;
    std::partial_sum(pos.begin(), pos.end(), pos.begin());
    for (int c = 0; c <= cols; c++)
      t_ai[c] = pos[c] + base;
    for (int i = 0; i < rows; i++)
      for (int k = ai[i] - base; k < ai[i + 1] - base; k++) {
        const int q = pos[aj[k] - base]++;
        t_aj[q] = i + base;
        if (vals)
          t_av[q] = av[k];
      }
    return;
  }
  // large: on the host's threads, in two stable passes.  (1) rows are cut
  // into T chunks of about equal entries; each chunk's entries go to column
  // blocks of 2^shift columns, blocks major, chunks in order -- so inside a
  // block the entries stay in row order.  (2) each block is counting-sorted by column
  // on its own (stable).  The result is the one-pass order exactly.
  const int T = std::max(1, omp_get_max_threads());
  int shift = 0; // column blocks of 2^shift columns, about 8 per thread
  while (((long long)cols >> shift) > 8LL * T)
    shift++;
  const int B = (int)(((long long)cols + (1LL << shift) - 1) >> shift);
  std::vector<int> r0(T + 1);
  for (int t = 0; t <= T; t++) {
    const long long want = (long long)nnz * t / T;
    r0[t] = (int)(std::lower_bound(ai, ai + rows + 1, (int)(want + base)) - ai);
  }
  r0[T] = rows;
  std::vector<long long> off((size_t)T * B, 0); // [chunk][block]: a chunk's own row
#pragma omp parallel for schedule(static, 1)
  for (int t = 0; t < T; t++) {
    long long *o = off.data() + (size_t)t * B;
    for (int k = ai[r0[t]] - base; k < ai[r0[t + 1]] - base; k++)
      o[(aj[k] - base) >> shift]++;
  }
  long long run = 0;
  std::vector<long long> bstart(B + 1);
  for (int b = 0; b < B; b++) {
    bstart[b] = run;
    for (int t = 0; t < T; t++) {
      const long long c = off[(size_t)t * B + b];
      off[(size_t)t * B + b] = run;
      run += c;
    }
  }
  bstart[B] = run;
  // scratch left uninitialised (every slot is written below), so its pages
  // are first touched by the threads that fill them
  std::unique_ptr<int[]> tc(new int[nnz]), tr(new int[nnz]);
  std::unique_ptr<double[]> tv(vals ? new double[nnz] : nullptr);
#pragma omp parallel for schedule(static, 1)
  for (int t = 0; t < T; t++)
    for (int i = r0[t]; i < r0[t + 1]; i++)
      for (int k = ai[i] - base; k < ai[i + 1] - base; k++) {
        const int c = aj[k] - base;
        const long long q = off[(size_t)t * B + (c >> shift)]++;
        tc[q] = c;
        tr[q] = i;
        if (vals)
          tv[q] = av[k];
      }
  t_ai[cols] = nnz + base;
#pragma omp parallel
  {
    std::vector<int> cnt;
#pragma omp for schedule(dynamic, 1)
    for (int b = 0; b < B; b++) {
      const int c0 = b << shift, c1 = (int)std::min<long long>(cols, (long long)(b + 1) << shift);
      cnt.assign(c1 - c0 + 1, 0);
      for (long long q = bstart[b]; q < bstart[b + 1]; q++)
        cnt[tc[q] - c0 + 1]++;
      for (int c = 0; c < c1 - c0; c++)
        cnt[c + 1] += cnt[c];
      for (int c = c0; c < c1; c++)
        t_ai[c] = (int)(bstart[b] + cnt[c - c0]) + base;
      for (long long q = bstart[b]; q < bstart[b + 1]; q++) {
        const long long w = bstart[b] + cnt[tc[q] - c0]++;
        t_aj[w] = tr[q] + base;
        if (vals)
          t_av[w] = tv[q];
      }
    }
  }
}

// matrix_utils.hpp:429-472 permute / :474-480 permuteRow: row i of the
// result is row iperm[i] of A, columns renamed through perm (if given) and
// each row re-sorted by column (the reference's insertion sort is stable
// for distinct columns, so any sort of distinct keys gives its order).
void permute(int n, int base, const int *ai, const int *aj, const double *av,
             const int *iperm, const int *perm, int *p_ai, int *p_aj,
             double *p_av) {
  p_ai[0] = base;
  for (int i = 0; i < n; i++) {
    const int src = iperm ? iperm[i] - base : i;
    p_ai[i + 1] = p_ai[i] + (ai[src + 1] - ai[src]);
  }
  // rows are independent once their starts are known: the host's threads
  // fill them (each row sorted on its own, so the result does not depend
  // on the threads)
#pragma omp parallel
  {
    std::vector<std::pair<int, double>> row;
#pragma omp for schedule(dynamic, 4096)
    for (int i = 0; i < n; i++) {
      const int src = iperm ? iperm[i] - base : i;
      const int o = p_ai[i] - base, s = ai[src] - base, len = ai[src + 1] - ai[src];
      if (!perm) {
        std::memcpy(p_aj + o, aj + s, sizeof(int) * len);
        std::memcpy(p_av + o, av + s, sizeof(double) * len);
        continue;
      }
      row.resize(len);
      for (int q = 0; q < len; q++)
        row[q] = {perm[aj[s + q] - base], av[s + q]};
      std::sort(row.begin(), row.end(),
                [](const auto &a, const auto &b) { return a.first < b.first; });
      for (int q = 0; q < len; q++) {
        p_aj[o + q] = row[q].first;
        p_av[o + q] = row[q].second;
      }
    }
  }
}

// matrix_utils.hpp:562-576 permuteVec: out[i] = v[iperm[i] - base] (a copy
// without iperm).
void permute_vec(int n, int base, const double *v, const int *iperm, double *out) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; i++)
    out[i] = v[iperm ? iperm[i] - base : i];
}

// utils.cpp:101-108 inversePermute: iperm[perm[i] - base] = i + base.
void inverse_permute(int n, int base, const int *perm, int *iperm) {
  for (int i = 0; i < n; i++)
    iperm[perm[i] - base] = i + base;
}

// matrix_utils.hpp:677-704 Diagonal: per row the first stored column not
// below the row (a binary search over the row's sorted columns); diagpos
// gets its position (with base), diag its value (inverted when asked, 0
// becoming 1).  Returns false when some row has no diagonal entry; that
// row's position is where the diagonal would go, and its value is what is
// stored there -- 0 past the last entry, where the reference reads beyond
// its arrays.
bool diagonal(int n, int base, const int *ai, const int *aj, const double *av, int *diagpos,
              double *diag, bool invert) {
  const int nnz = ai[n] - base;
  bool all = true;
  for (int i = 0; i < n; i++) {
    const int *lo = aj + ai[i] - base, *hi = aj + ai[i + 1] - base;
    const int *at = std::lower_bound(lo, hi, i + base);
    const int k = (int)(at - aj);
    if (at == hi || *at != i + base)
      all = false;
    if (diagpos)
      diagpos[i] = k + base;
    if (diag) {
      double v = k < nnz ? av[k] : 0.0;
      if (invert)
        v = v == 0 ? 1.0 : 1.0 / v;
      diag[i] = v;
    }
  }
  return all;
}

// ILU(0) on A's own pattern (no reference routine: the reference factors ILU
// through MKL, and its own level-0 path never fills the upper-part
// positions, incomplete_lu.cpp:166 / :267-269).  Row by row (IKJ order): for
// each stored k < i, ascending, l_ik = a_ik / u_kk, then a_ij -= l_ik * u_kj
// for every stored j > k that row k also holds.  The result, in A's pattern,
// is the strictly lower L (unit diagonal implied) and U with its diagonal --
// what SplitLDU splits and the unit-lower / upper solves apply
// (incomplete_lu.cpp:36-48).  Returns the first row whose pivot is zero, or
// -1; -2 when a row has no diagonal entry.
int ilu0(int n, int base, const int *ai, const int *aj, const double *av, double *lu) {
  const int nnz = ai[n] - base;
  std::memcpy(lu, av, sizeof(double) * (size_t)nnz);
  std::vector<int> diag(n), where(n, -1);
  for (int i = 0; i < n; i++) {
    const int *lo = aj + ai[i] - base, *hi = aj + ai[i + 1] - base;
    const int *at = std::lower_bound(lo, hi, i + base);
    if (at == hi || *at != i + base)
      return -2;
    diag[i] = (int)(at - aj);
  }
  for (int i = 0; i < n; i++) {
    const int r0 = ai[i] - base, r1 = ai[i + 1] - base;
    for (int k = r0; k < r1; k++)
      where[aj[k] - base] = k;
    for (int k = r0; k < diag[i]; k++) {
      const int c = aj[k] - base; // c < i
      const double piv = lu[diag[c]];
      if (piv == 0.0)
        return c;
      lu[k] /= piv;
      const double l = lu[k];
      for (int m = diag[c] + 1; m < ai[c + 1] - base; m++) {
        const int w = where[aj[m] - base];
        if (w >= 0)
          lu[w] -= l * lu[m];
      }
    }
    if (lu[diag[i]] == 0.0)
      return i;
    for (int k = r0; k < r1; k++)
      where[aj[k] - base] = -1;
  }
  return -1;
}

// matrix_utils.hpp:720-803 SplitLDU: strict lower, diagonal (0 when
// missing), strict upper; entries keep their column order.
void split_ldu(int n, int base, const int *ai, const int *aj, const double *av,
               int *l_ai, int *l_aj, double *l_av, double *d, int *u_ai,
               int *u_aj, double *u_av, int *lnnz, int *unnz) {
  // rows are independent once their output starts are known: counted and
  // filled on the host's threads (the same arrays as one pass in row order)
  l_ai[0] = base;
  u_ai[0] = base;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; i++) {
    int lc = 0, uc = 0;
    for (int k = ai[i] - base; k < ai[i + 1] - base; k++) {
      const int c = aj[k] - base;
      lc += c < i;
      uc += c > i;
    }
    l_ai[i + 1] = lc;
    u_ai[i + 1] = uc;
  }
  for (int i = 0; i < n; i++) {
    l_ai[i + 1] += l_ai[i];
    u_ai[i + 1] += u_ai[i];
  }
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; i++) {
    int lp = l_ai[i] - base, up = u_ai[i] - base;
    d[i] = 0;
    for (int k = ai[i] - base; k < ai[i + 1] - base; k++) {
      const int c = aj[k] - base;
      if (c < i) {
        l_aj[lp] = aj[k];
        l_av[lp++] = av[k];
      } else if (c > i) {
        u_aj[up] = aj[k];
        u_av[up++] = av[k];
      } else {
        d[i] = av[k];
      }
    }
  }
  *lnnz = l_ai[n] - base;
  *unnz = u_ai[n] - base;
}

// matrix_utils.hpp:805-879 SplitTriangle<L|U>: the triangle incl. diagonal.
int split_triangle(int uplo, int n, int base, const int *ai, const int *aj,
                   const double *av, int *t_ai, int *t_aj, double *t_av) {
  auto keep = [uplo](int c, int i) { return uplo == LA_UPPER ? c >= i : c <= i; };
  t_ai[0] = base;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; i++) {
    int cnt = 0;
    for (int k = ai[i] - base; k < ai[i + 1] - base; k++)
      cnt += keep(aj[k] - base, i);
    t_ai[i + 1] = cnt;
  }
  for (int i = 0; i < n; i++)
    t_ai[i + 1] += t_ai[i];
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; i++) {
    int p = t_ai[i] - base;
    for (int k = ai[i] - base; k < ai[i + 1] - base; k++)
      if (keep(aj[k] - base, i)) {
        t_aj[p] = aj[k];
        t_av[p++] = av[k];
      }
  }
  return t_ai[n] - base;
}

// precond.hpp:615-693 ICCLevelNumeric on the IC(0) pattern (the upper
// triangle with the diagonal first in each row; precond.hpp:13-37).
//
// Up-looking factorisation.  Row j of U starts as row j of A with the
// diagonal scaled by (1 + omega).  The earlier rows k that hold an entry in
// column j are found through per-column lists threaded through `next`:
// after row k is finished (and each time one of its entries is consumed),
// k is pushed on the list of the column of its next unconsumed entry, with
// `cursor[k]` pointing at that entry.  The lists are LIFO, and the updates
// are applied in list order, which is the reference's order; each update
// subtracts U_kj * U_k,c from the matching entries c of row j.  Finally the
// pivot p is checked (p < 0: breakdown) and U_jj = sqrt(p), U_jc /= U_jj.
bool icc0(int n, int base, const int *u_ai, const int *u_aj, const double *u_av,
          double omega, double *icc_av) {
  constexpr int kEnd = INT_MAX;
  std::vector<int> next(n, kEnd), cursor(n, 0);
  for (int j = 0; j < n; j++) {
    const int rs = u_ai[j] - base, re = u_ai[j + 1] - base;
    icc_av[rs] = u_av[rs] * (1.0 + omega);
    std::memcpy(icc_av + rs + 1, u_av + rs + 1, sizeof(double) * (re - rs - 1));
    for (int k = next[j]; k < j;) {
      int ck = cursor[k]++;
      const int ke = u_ai[k + 1] - base;
      const int after = next[k];
      if (ck + 1 < ke) { // push k on the list of its next column
        const int c = u_aj[ck + 1] - base;
        next[k] = next[c];
        next[c] = k;
      }
      const double ukj = icc_av[ck];
      for (int p = rs; ck < ke && p < re;) {
        if (u_aj[ck] == u_aj[p])
          icc_av[p++] -= ukj * icc_av[ck++];
        else if (u_aj[ck] < u_aj[p])
          ck++;
        else
          p++;
      }
      k = after;
    }
    if (re - rs > 1) {
      const int c = u_aj[rs + 1] - base;
      next[j] = next[c];
      next[c] = j;
      cursor[j] = rs + 1;
    }
    if (icc_av[rs] < 0)
      return false;
    const double piv = std::sqrt(icc_av[rs]);
    icc_av[rs] = piv;
    for (int p = rs + 1; p < re; p++)
      icc_av[p] /= piv;
  }
  return true;
}

// reordering/Reordering.cpp:37-136 SerialCM (reverse Cuthill-McKee).
//
// Components: the reference's union-find links toward the larger index, so
// each component's root is its largest node; components are visited in
// ascending root order and their members in ascending index order
// (reordering/UnionFind.cpp:83-129, 217-293).  Components of one or two
// nodes are emitted as is.  Otherwise a pseudo-peripheral source is chosen
// as the reference executes PseudoDiameter (reordering/Reordering.h:72-136):
// start at the first node of minimum degree; BFS from it; greedily take up
// to five last-level candidates by (degree, index), setting the degree of
// each candidate and of its neighbours to INT_MAX (a persistent change that
// later breaks the CM ties); BFS from the first candidate -- deeper: it
// becomes the source and the search repeats; otherwise the search stops.
// The CM sweep visits the ordering level by level and appends, for each
// node, its unvisited neighbours of the next BFS level sorted by (degree,
// index).  The complete ordering is reversed; perm is its inverse.
namespace {
struct Bfs {
  const int *ai, *aj;
  int base;
  std::vector<int> level, queue;
  std::vector<std::vector<int>> found; // per-thread finds of one frontier
  // BFS from src over its component; returns the level count.  Level by
  // level: a large frontier is split over the host's threads, which claim a
  // vertex by a compare-and-swap on its level.  The levels, and the set of
  // vertices on each, are those of the sequential search; only the order
  // inside a level may differ, and rcm() never depends on it.  Only the
  // vertices the previous run reached are reset, so a pattern with many
  // components is not O(n) per component.
  int run(int n, int src) {
    if ((int)level.size() != n)
      level.assign(n, -1);
    else
      for (int v : queue)
        level[v] = -1;
    queue.clear();
    queue.push_back(src);
    level[src] = 0;
    for (size_t head = 0; head < queue.size();) {
      const size_t begin = head, end = queue.size();
      const int lev = level[queue[begin]] + 1;
      head = end;
      if (end - begin < 4096) {
        for (size_t h = begin; h < end; h++)
          for (int k = ai[queue[h]] - base; k < ai[queue[h] + 1] - base; k++) {
            const int v = aj[k] - base;
            if (level[v] < 0) {
              level[v] = lev;
              queue.push_back(v);
            }
          }
        continue;
      }
#pragma omp parallel
      {
#pragma omp single
        found.assign(omp_get_num_threads(), {});
        std::vector<int> &mine = found[omp_get_thread_num()];
#pragma omp for schedule(static)
        for (long long h = (long long)begin; h < (long long)end; h++)
          for (int k = ai[queue[h]] - base; k < ai[queue[h] + 1] - base; k++) {
            int *lv = &level[aj[k] - base];
            int expect = -1;
            if (__atomic_load_n(lv, __ATOMIC_RELAXED) < 0 &&
                __atomic_compare_exchange_n(lv, &expect, lev, false, __ATOMIC_RELAXED,
                                            __ATOMIC_RELAXED))
              mine.push_back(aj[k] - base);
          }
      }
      for (const std::vector<int> &f : found)
        queue.insert(queue.end(), f.begin(), f.end());
    }
    return level[queue.back()] + 1;
  }
};
} // namespace

// With `device`, components of at least kRcmDeviceMin nodes are ordered on
// the GPU (la_rcm.cu; same ordering) when no row holds more than
// kRcmMaxDegree entries.
la_status rcm(int n, int base, const int *ai, const int *aj, int *iperm, int *perm,
              bool device) {
  std::vector<int> deg(n);
  int maxdeg = 0;
  for (int i = 0; i < n; i++) {
    deg[i] = ai[i + 1] - ai[i];
    maxdeg = std::max(maxdeg, deg[i]);
  }
  device = device && maxdeg <= kRcmMaxDegree;
  struct DeviceOwner {
    RcmDevice *d = nullptr;
    ~DeviceOwner() { rcm_device_destroy(d); }
  } dev;
  Bfs bfs{ai, aj, base, {}, {}, {}};

  // components, ordered by their largest node; members ascending
  std::vector<int> comp(n, -1), comp_max;
  for (int i = 0; i < n; i++) {
    if (comp[i] >= 0)
      continue;
    const int id = (int)comp_max.size();
    bfs.run(n, i);
    int mx = i;
    for (int v : bfs.queue) {
      comp[v] = id;
      mx = std::max(mx, v);
    }
    comp_max.push_back(mx);
  }
  const int ncomp = (int)comp_max.size();
  std::vector<int> rank(ncomp), start(ncomp + 1, 0), members(n);
  {
    int r = 0;
    for (int i = 0; i < n; i++)
      if (comp_max[comp[i]] == i)
        rank[comp[i]] = r++;
    for (int i = 0; i < n; i++)
      start[rank[comp[i]] + 1]++;
    std::partial_sum(start.begin(), start.end(), start.begin());
    std::vector<int> fill(start.begin(), start.end() - 1);
    for (int i = 0; i < n; i++)
      members[fill[rank[comp[i]]]++] = i;
  }

  std::vector<int> children;
  for (int c = 0; c < ncomp; c++) {
    const int off = start[c], size = start[c + 1] - start[c];
    if (size <= 2) {
      for (int q = 0; q < size; q++)
        iperm[off + q] = members[off + q] + base;
      continue;
    }
    if (device && size >= kRcmDeviceMin) {
      if (!dev.d) {
        la_status st = LA_OK;
        dev.d = rcm_device_create(n, base, ai, aj, deg.data(), &st);
        if (!dev.d)
          return st;
      }
      LA_TRY(rcm_device_component(dev.d, members.data() + off, size, iperm + off));
      continue;
    }
    int src = members[off];
    for (int q = off; q < off + size; q++)
      if (deg[members[q]] < deg[src])
        src = members[q];
    for (;;) {
      const int height = bfs.run(n, src);
      std::vector<int> last;
      for (int v : bfs.queue)
        if (bfs.level[v] == height - 1)
          last.push_back(v);
      int first = -1;
      for (int chosen = 0; chosen < 5; chosen++) {
        int sel = -1;
        for (int v : last)
          if (deg[v] != INT_MAX &&
              (sel < 0 || deg[v] < deg[sel] || (deg[v] == deg[sel] && v < sel)))
            sel = v;
        if (sel < 0)
          break;
        if (first < 0)
          first = sel;
        deg[sel] = INT_MAX;
        for (int k = ai[sel] - base; k < ai[sel + 1] - base; k++)
          deg[aj[k] - base] = INT_MAX;
      }
      if (first < 0 || bfs.run(n, first) <= height)
        break;
      src = first;
    }
    // Cuthill-McKee sweep
    const int height = bfs.run(n, src);
    std::vector<int> lstart(height + 1, 0);
    for (int q = off; q < off + size; q++)
      lstart[bfs.level[members[q]] + 1]++;
    std::partial_sum(lstart.begin(), lstart.end(), lstart.begin());
    int e = off;
    iperm[e++] = src + base;
    auto by_deg = [&](int a, int b) {
      return deg[a] != deg[b] ? deg[a] < deg[b] : a < b;
    };
    for (int l = 0; l < height; l++)
      for (int r = lstart[l]; r < lstart[l + 1]; r++) {
        const int u = iperm[off + r] - base;
        children.clear();
        for (int k = ai[u] - base; k < ai[u + 1] - base; k++) {
          const int v = aj[k] - base;
          if (bfs.level[v] == l + 1) {
            children.push_back(v);
            bfs.level[v] = -1;
          }
        }
        std::sort(children.begin(), children.end(), by_deg);
        for (int v : children)
          iperm[e++] = v + base;
      }
  }
  std::reverse(iperm, iperm + n);
  for (int i = 0; i < n; i++)
    perm[iperm[i] - base] = i + base;
  return LA_OK;
}

} // namespace la
