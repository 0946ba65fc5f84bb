// la_partition.cpp -- row partition for the partitioned triangular solve.
//
// Goal: parts whose dependency graph (part A -> part B when a row of B reads
// a row of A) is acyclic and shallow, so that a dependency path crosses few
// part boundaries.  Every cut is made on a coordinate f that is monotone
// along the dependency edges (f(j) <= f(i) whenever row i reads row j), low
// values to one side, high values to the other: an edge can then only cross
// from the low side to the high side, so ordering the parts low-before-high
// at every cut makes every cross-part edge go forward (acyclic), and a path
// crosses each cut at most once.  Cutting P ways along ONE coordinate (say
// the level) gives P slabs that a path crosses P - 1 times; cutting along
// three independent monotone coordinates gives boxes, crossed about
// 3 * P^(1/3) times.
//
// Coordinates: differences of breadth-first distances to landmark vertices,
// d_a - d_b, kept when monotone along every dependency edge; the level is
// always a candidate.  Landmarks are spread by farthest-point sampling over
// the vertices of minimum degree (the corners of a mesh: on a grid, corner
// landmarks make d_a - d_b a multiple of one grid axis).  Among the monotone
// candidates, the narrowest are taken first, each only if it is independent
// enough of those already taken (Gram-Schmidt residual), up to three.  The
// parts then come from a k-d tree: each node is cut on the candidate with
// the largest span over its rows, at the value that best splits its rows in
// the ratio of the part counts of its two halves.
//
// This is scheduling, not arithmetic: the triangular solve computes every
// row with the same operations whatever the partition.

#include "la_internal.h"

#include <algorithm>
#include <climits>
#include <cmath>
#include <functional>
#include <numeric>
#include <vector>

namespace la {
namespace {

// Breadth-first distances from src (-1 where unreachable); returns the
// number of vertices reached.  Level-synchronous: the host's threads split
// each frontier and claim a vertex by a compare-and-swap on its distance, so
// the distances are those of the sequential search whatever the threads'
// order (only the order of a frontier varies, and nothing reads it).
int bfs_dist(int n, const int *xadj, const int *adj, int src, std::vector<int> &d) {
  d.assign(n, -1);
  d[src] = 0;
  std::vector<int> frontier{src}, next;
  int reached = 1;
  for (int level = 1; !frontier.empty(); level++) {
    next.clear();
    const int fs = (int)frontier.size();
    if (fs < 4096) { // small frontier: no threads
      for (int f = 0; f < fs; f++)
        for (int k = xadj[frontier[f]]; k < xadj[frontier[f] + 1]; k++)
          if (d[adj[k]] < 0) {
            d[adj[k]] = level;
            next.push_back(adj[k]);
          }
    } else {
#pragma omp parallel
      {
        std::vector<int> mine;
#pragma omp for schedule(static) nowait
        for (int f = 0; f < fs; f++)
          for (int k = xadj[frontier[f]]; k < xadj[frontier[f] + 1]; k++) {
            int *dv = &d[adj[k]];
            int expect = -1;
            if (__atomic_load_n(dv, __ATOMIC_RELAXED) < 0 &&
                __atomic_compare_exchange_n(dv, &expect, level, false, __ATOMIC_RELAXED,
                                            __ATOMIC_RELAXED))
              mine.push_back(adj[k]);
          }
#pragma omp critical
        next.insert(next.end(), mine.begin(), mine.end());
      }
    }
    reached += (int)next.size();
    frontier.swap(next);
  }
  return reached;
}

} // namespace

// Vertex v's neighbours: its own row's columns, then the rows that store v
// (the transpose's row v, ascending), both 0-based; built on the host's
// threads from the transpose.
void undirected_pattern(int n, int base, const int *ai, const int *aj, std::vector<int> &xadj,
                        std::vector<int> &adj) {
  const int nnz = ai[n] - base;
  std::vector<int> t_ai(n + 1), t_aj(std::max(nnz, 1));
  transpose(n, n, base, ai, aj, nullptr, t_ai.data(), t_aj.data(), nullptr);
  xadj.assign(n + 1, 0);
  adj.resize(2 * (size_t)nnz);
  for (int v = 0; v < n; v++)
    xadj[v + 1] = xadj[v] + (ai[v + 1] - ai[v]) + (t_ai[v + 1] - t_ai[v]);
#pragma omp parallel for schedule(dynamic, 4096)
  for (int v = 0; v < n; v++) {
    int w = xadj[v];
    for (int k = ai[v] - base; k < ai[v + 1] - base; k++)
      adj[w++] = aj[k] - base;
    for (int k = t_ai[v] - base; k < t_ai[v + 1] - base; k++)
      adj[w++] = t_aj[k] - base;
  }
}

namespace {

// The stage after the landmark candidates: the level coordinate joins them,
// the narrowest independent ones are chosen, and the k-d cuts are made.
// coordinate(c, f) writes candidate c's values (c.a >= 0) into f and
// returns false if it could not.  Returns the coordinates used, -1 on such
// a failure.
int cut_parts(int n, const int *lvl, int nparts, int *part, std::vector<PartitionCand> cands,
              const std::function<bool(const PartitionCand &, std::vector<int> &)> &coordinate) {
  using Cand = PartitionCand;
  {
    int lo = INT_MAX, hi = INT_MIN;
    for (int v = 0; v < n; v++) {
      lo = std::min(lo, lvl[v]);
      hi = std::max(hi, lvl[v]);
    }
    cands.push_back({-1, -1, 1, (long long)hi - lo});
    std::stable_sort(cands.begin(), cands.end(),
                     [](const Cand &x, const Cand &y) { return x.range < y.range; });
  }
  std::vector<std::vector<int>> coords; // chosen coordinates
  std::vector<std::vector<double>> basis;
  // greedy selection: narrowest first, each with a Gram-Schmidt residual of
  // at least half its norm against those already chosen.  The sums run over
  // fixed 64K-vertex chunks on the host's threads and add the chunks' sums in
  // chunk order, so they do not depend on the number of threads.
  auto chunked_sum = [n](auto term) {
    constexpr int kChunk = 1 << 16;
    const int nc = (n + kChunk - 1) / kChunk;
    std::vector<double> part(nc);
#pragma omp parallel for schedule(static)
    for (int c = 0; c < nc; c++) {
      double s = 0;
      for (int v = c * kChunk; v < std::min(n, (c + 1) * kChunk); v++)
        s += term(v);
      part[c] = s;
    }
    double s = 0;
    for (double x : part)
      s += x;
    return s;
  };
  for (const Cand &c : cands) {
    if (coords.size() == 3)
      break;
    std::vector<int> f(n);
    if (c.a < 0)
      std::copy(lvl, lvl + n, f.begin());
    else if (!coordinate(c, f))
      return -1;
    long long fsum = 0; // integer: exact in any order
#pragma omp parallel for schedule(static) reduction(+ : fsum)
    for (int v = 0; v < n; v++)
      fsum += f[v];
    const double mean = (double)fsum / n;
    const double var =
        chunked_sum([&](int v) { return (f[v] - mean) * (f[v] - mean); }) / n;
    if (var <= 0)
      continue;
    const double sd = std::sqrt(var);
    std::vector<double> r(n);
#pragma omp parallel for schedule(static)
    for (int v = 0; v < n; v++)
      r[v] = (f[v] - mean) / sd;
    for (const std::vector<double> &q : basis) {
      const double dot = chunked_sum([&](int v) { return r[v] * q[v]; }) / n;
#pragma omp parallel for schedule(static)
      for (int v = 0; v < n; v++)
        r[v] -= dot * q[v];
    }
    const double nr = std::sqrt(chunked_sum([&](int v) { return r[v] * r[v]; }) / n);
    if (nr < 0.5)
      continue;
#pragma omp parallel for schedule(static)
    for (int v = 0; v < n; v++)
      r[v] /= nr;
    basis.push_back(std::move(r));
    coords.push_back(std::move(f));
  }
  basis.clear();

  // k-d tree of value-threshold cuts; the two halves of a node are cut as
  // independent tasks on the host's threads (disjoint ranges of `order`)
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::function<void(int, int, int, int)> split = [&](int lo, int hi, int k, int p0) {
    if (k == 1 || hi - lo <= 1) {
      for (int q = lo; q < hi; q++)
        part[order[q]] = p0;
      // a single row split further leaves parts empty
      return;
    }
    const int k1 = k / 2;
    const long long want = (long long)(hi - lo) * k1 / k;
    // coordinates by span, widest first; take the first that splits
    std::vector<std::pair<long long, int>> spans;
    std::vector<int> lows;
    for (int a = 0; a < (int)coords.size(); a++) {
      int mn = INT_MAX, mx = INT_MIN;
      for (int q = lo; q < hi; q++) {
        const int f = coords[a][order[q]];
        mn = std::min(mn, f);
        mx = std::max(mx, f);
      }
      spans.push_back({(long long)mx - mn, a});
      lows.push_back(mn);
    }
    std::stable_sort(spans.begin(), spans.end(),
                     [](auto &x, auto &y) { return x.first > y.first; });
    int cut = -1;
    std::vector<long long> hist;
    for (const auto &sa : spans) {
      if (sa.first == 0)
        break;
      const std::vector<int> &f = coords[sa.second];
      const int mn = lows[sa.second];
      // histogram of the node's values; the threshold keeps f < thr low
      hist.assign((size_t)sa.first + 2, 0);
      for (int q = lo; q < hi; q++)
        hist[f[order[q]] - mn]++;
      long long below = 0, bdev = LLONG_MAX;
      int thr = 0;
      bool found = false;
      for (size_t v = 1; v < hist.size(); v++) {
        below += hist[v - 1];
        if (hist[v] == 0 && v + 1 < hist.size())
          continue; // only thresholds just below a present value
        const long long dev = std::llabs(below - want);
        if (below > 0 && below < hi - lo && dev < bdev) {
          bdev = dev;
          thr = mn + (int)v;
          found = true;
        }
      }
      if (!found)
        continue;
      const auto mid = std::stable_partition(order.begin() + lo, order.begin() + hi,
                                             [&](int v) { return f[v] < thr; });
      cut = (int)(mid - order.begin());
      break;
    }
    if (cut < 0) { // no coordinate separates these rows: keep them together
      for (int q = lo; q < hi; q++)
        part[order[q]] = p0;
      return;
    }
    if (hi - lo >= (1 << 15)) {
#pragma omp task shared(split)
      split(lo, cut, k1, p0);
#pragma omp task shared(split)
      split(cut, hi, k - k1, p0 + k1);
#pragma omp taskwait
    } else {
      split(lo, cut, k1, p0);
      split(cut, hi, k - k1, p0 + k1);
    }
  };
#pragma omp parallel
#pragma omp single
  split(0, n, std::max(1, nparts), 0);
  return (int)coords.size();
}

} // namespace

int monotone_partition(int n, const int *xadj, const int *adj, const int *dep_ptr,
                       const int *dep_col, int base, const int *lvl, int nparts, int *part) {
  if (n == 0)
    return 0;
  auto search = [&](int src, std::vector<int> &d) { return bfs_dist(n, xadj, adj, src, d); };
  std::vector<PartitionCand> cands;
  std::vector<std::vector<int>> dist;
  {
    int dmin = INT_MAX;
    for (int v = 0; v < n; v++)
      dmin = std::min(dmin, xadj[v + 1] - xadj[v]);
    std::vector<int> low;
    for (int v = 0; v < n; v++)
      if (xadj[v + 1] - xadj[v] == dmin)
        low.push_back(v);
    std::vector<int> d, mind;
    bool connected = search(low[0], d) == n;
    if (connected) {
      dist.push_back(d);
      mind = d;
      while (dist.size() < 8) {
        int best = -1;
        for (int v : low)
          if (best < 0 || mind[v] > mind[best])
            best = v;
        if (best < 0 || mind[best] == 0)
          break;
        search(best, d);
        dist.push_back(d);
#pragma omp parallel for schedule(static)
        for (int v = 0; v < n; v++)
          mind[v] = std::min(mind[v], d[v]);
      }
    }
    // landmark pairs, checked on the host's threads (integer work: the same
    // candidates, kept in pair order, whatever the threads)
    const int L = (int)dist.size();
    std::vector<std::pair<int, int>> pairs;
    for (int a = 0; a < L; a++)
      for (int b = a + 1; b < L; b++)
        pairs.push_back({a, b});
    const int np = (int)pairs.size();
    std::vector<PartitionCand> found(np);
    std::vector<char> keep(np, 0);
#pragma omp parallel for schedule(dynamic)
    for (int q = 0; q < np; q++) {
      const int a = pairs[q].first, b = pairs[q].second;
      const std::vector<int> &da = dist[a], &db = dist[b];
      long long pos = 0, neg = 0;
      for (int i = 0; i < n && !(pos && neg); i++)
        for (int k = dep_ptr[i] - base; k < dep_ptr[i + 1] - base; k++) {
          const int j = dep_col[k] - base;
          const int df = (da[i] - db[i]) - (da[j] - db[j]);
          pos += df > 0;
          neg += df < 0;
        }
      if ((pos == 0) == (neg == 0))
        continue; // not monotone, or constant along every edge
      int lo = INT_MAX, hi = INT_MIN;
      for (int v = 0; v < n; v++) {
        const int f = da[v] - db[v];
        lo = std::min(lo, f);
        hi = std::max(hi, f);
      }
      found[q] = {a, b, pos > 0 ? 1 : -1, (long long)hi - lo};
      keep[q] = 1;
    }
    for (int q = 0; q < np; q++)
      if (keep[q])
        cands.push_back(found[q]);
  }
  return cut_parts(n, lvl, nparts, part, cands,
                   [&](const PartitionCand &c, std::vector<int> &f) {
#pragma omp parallel for schedule(static)
                     for (int v = 0; v < n; v++)
                       f[v] = c.sign * (dist[c.a][v] - dist[c.b][v]);
                     return true;
                   });
}

int monotone_partition_device(int n, int base, const int *ai, const int *aj, const int *lvl,
                              int nparts, int *part, la_status *st) {
  *st = LA_OK;
  if (n == 0)
    return 0;
  LandmarksDevice *M = landmarks_device_create(n, base, ai, aj, st);
  if (!M)
    return -1;
  struct Owner {
    LandmarksDevice *m;
    ~Owner() { landmarks_device_destroy(m); }
  } own{M};
  std::vector<PartitionCand> cands;
  if ((*st = landmarks_device_candidates(M, cands)) != LA_OK)
    return -1;
  const int used = cut_parts(n, lvl, nparts, part, cands,
                             [&](const PartitionCand &c, std::vector<int> &f) {
                               *st = landmarks_device_coordinate(M, c, f.data());
                               return *st == LA_OK;
                             });
  return used;
}

} // namespace la
