// la_factor.cu -- IC(0) and ILU(0) numeric factorisation on the GPU.
//
// Reference: ICCLevel0SymSymbolic + ICCLevelNumeric (sparse_mat_op/
// precond.hpp:13-37, 615-693), the up-looking IC(0) whose factor U (the
// upper triangle of A, diagonal first in each row) gives A ~= U^T U, with
// the shift-retry loop of incomplete_cholesky_k_2 (mkl_wrapper/
// incomplete_cholesky.cpp:286-342); and ILU(0) on A's own pattern in IKJ
// order (the reference factors ILU through MKL, incomplete_lu.cpp:277-325;
// the host restatement here is la_host.cpp's ilu0).
//
// B200 design.  The factorisation is split into a symbolic plan, built once
// per pattern on the host, and a numeric pass on the GPU that can run many
// times (new values, or the shift retries after a breakdown):
//  * symbolic: the host records, for every row j, the ordered list of
//    updates it receives -- for IC(0) the rows k with U_kj != 0 in the order
//    the up-looking algorithm's linked lists deliver them (a rule on the
//    pattern alone, update_before, applied to each row in parallel), for
//    ILU(0) the stored k < j in ascending order -- and, for each update, the
//    (target entry of row j, source entry of row k) pairs it subtracts.  Row j depends exactly
//    on the rows of its updates, so their level sets (by longest path, as
//    TopologicalSort2 computes them) order the rows for the device;
//  * numeric: one persistent launch; warps claim 32-row chunks in level
//    order from an atomic ticket, one lane per row.  A lane copies its row's
//    values, waits (bounded by the global timer) for each update's source row
//    to be published, applies the update's products with exact, never fused
//    multiplies and subtractions in the recorded order, finishes its row
//    (IC: pivot check, square root, row division; ILU: zero-pivot check) and
//    publishes it.  Every value is produced by the same operations in the
//    same order as the host algorithm: the factor is bit-identical to it.
//    Because a chunk is claimed only after every earlier chunk, the lowest
//    unfinished row always has its inputs, and the pass cannot deadlock.
// A breakdown (IC: negative pivot; ILU: zero pivot) is reported as the
// smallest such row -- the row where the sequential algorithm stops, since
// no earlier row depends on a later one.
//
// Roofline: latency-bound (levels x one dependency round trip through L2);
// bytes per factorisation: nnz * 8 (values in) + nnz * 8 (factor out) +
// the update and pair lists (4 bytes per index).

#include "la_device.cuh"
#include "la_internal.h"

#include <algorithm>
#include <cstdlib>
#include <cmath>
#include <memory>
#include <vector>

namespace la {
namespace {

constexpr int kFactorThreads = 256;
constexpr int kFactorChunk = 32;
constexpr unsigned long long kFactorWaitNs = 1000000000ull; // 1 s
constexpr int kGroup = 8; // flags polled / pair sources loaded together
// pause between polls of unpublished rows (none: 64 / 256 ns measured no
// faster on the 128^3 and 192^3 factors, 2% faster on the 27-point one)
constexpr int kPollSleepNs = 0;

enum FactorKind { kIC0 = 0, kILU0 = 1 };

} // namespace
} // namespace la


namespace la {
namespace {

// The pattern's update lists.  IC(0): la_host.cpp's icc0 (the reference's
// ICCLevelNumeric order) replayed without arithmetic.  ILU(0): ilu0's IKJ
// loop replayed likewise.
struct Symbolic {
  std::vector<int> uptr, uk, us, upiv, pptr, ptgt, psrc, diag;
};

// The (target entry of row j, source entry of row k) pairs of one update:
// the columns row k holds from entry ck0 on that row j also holds.  Calls
// emit(p, ck) per pair, in ascending column order.
template <typename F>
inline void merge_pairs(const int *aj, int rs, int re, int ck0, int ke, F emit) {
  for (int p = rs, ck = ck0; ck < ke && p < re;) {
    if (aj[ck] == aj[p])
      emit(p++, ck++);
    else if (aj[ck] < aj[p])
      ck++;
    else
      p++;
  }
}

// Whether update x precedes update y in the list of the row they both
// update.  The up-looking algorithm keeps a LIFO list per row: row k joins
// row c's list when its cursor reaches column c, which happens while row r =
// the column before c in row k is processed (r = k for k's first
// off-diagonal; row k itself joins last, after r's own updates were
// delivered).  So a list holds its rows by descending r; among rows with the
// same r, row r itself first, then the updates of row r in the reverse of
// the order row r received them -- the same rule one column further back,
// with the direction flipped.  px / py: the entries before the target
// column in rows x and y; lx / ly: their diagonal entries.
inline bool update_before(const int *aj, int px, int lx, int py, int ly) {
  for (bool flip = false;; flip = !flip) {
    const int cx = aj[px], cy = aj[py];
    if (cx != cy)
      return (cx > cy) != flip;
    if (px == lx) // x is row cx itself
      return !flip;
    if (py == ly)
      return flip;
    px--;
    py--;
  }
}

// Row j receives one update per strict upper entry (k, j) of its column, in
// the order of its list (update_before), found per row in parallel; each
// update's (target, source) pairs are then merged in parallel, counted first
// and written second.  The rows' columns must ascend (checked by the caller).
void symbolic_ic0(int n, int base, const int *ai, const int *aj, Symbolic &S) {
  S.uptr.assign(n + 1, 0);
  S.diag.resize(n);
  for (int j = 0; j < n; j++)
    S.diag[j] = ai[j] - base;
  for (int k = 0; k < n; k++)
    for (int e = ai[k] - base + 1; e < ai[k + 1] - base; e++)
      S.uptr[aj[e] - base + 1]++;
  for (int j = 0; j < n; j++)
    S.uptr[j + 1] += S.uptr[j];
  const int nu = S.uptr[n];
  S.uk.resize(nu);
  S.us.resize(nu);
  {
    std::vector<int> fill(S.uptr.begin(), S.uptr.end() - 1);
    for (int k = 0; k < n; k++)
      for (int e = ai[k] - base + 1; e < ai[k + 1] - base; e++) {
        const int w = fill[aj[e] - base]++;
        S.uk[w] = k;
        S.us[w] = e;
      }
  }
#pragma omp parallel
  {
    std::vector<std::pair<int, int>> t; // (entry, row) of one row's updates
#pragma omp for schedule(dynamic, 4096)
    for (int j = 0; j < n; j++) {
      const int u0 = S.uptr[j], u1 = S.uptr[j + 1];
      if (u1 - u0 < 2)
        continue;
      t.clear();
      for (int u = u0; u < u1; u++)
        t.emplace_back(S.us[u], S.uk[u]);
      std::sort(t.begin(), t.end(), [&](const std::pair<int, int> &x,
                                        const std::pair<int, int> &y) {
        return update_before(aj, x.first - 1, ai[x.second] - base, y.first - 1,
                             ai[y.second] - base);
      });
      for (int u = u0; u < u1; u++) {
        S.us[u] = t[u - u0].first;
        S.uk[u] = t[u - u0].second;
      }
    }
  }
  S.pptr.assign((size_t)nu + 1, 0);
#pragma omp parallel for schedule(dynamic, 4096)
  for (int j = 0; j < n; j++) {
    const int rs = ai[j] - base, re = ai[j + 1] - base;
    for (int u = S.uptr[j]; u < S.uptr[j + 1]; u++) {
      int c = 0;
      merge_pairs(aj, rs, re, S.us[u], ai[S.uk[u] + 1] - base, [&](int, int) { c++; });
      S.pptr[u + 1] = c;
    }
  }
  for (int u = 0; u < nu; u++)
    S.pptr[u + 1] += S.pptr[u];
  S.ptgt.resize(S.pptr[nu]);
  S.psrc.resize(S.pptr[nu]);
#pragma omp parallel for schedule(dynamic, 4096)
  for (int j = 0; j < n; j++) {
    const int rs = ai[j] - base, re = ai[j + 1] - base;
    for (int u = S.uptr[j]; u < S.uptr[j + 1]; u++) {
      int w = S.pptr[u];
      merge_pairs(aj, rs, re, S.us[u], ai[S.uk[u] + 1] - base, [&](int p, int ck) {
        S.ptgt[w] = p;
        S.psrc[w++] = ck;
      });
    }
  }
}

void symbolic_ilu0(int n, int base, const int *ai, const int *aj, const std::vector<int> &diag,
                   Symbolic &S) {
  std::vector<int> where(n, -1);
  S.uptr.assign(n + 1, 0);
  S.pptr.assign(1, 0);
  S.diag = diag;
  for (int i = 0; i < n; i++) {
    const int r0 = ai[i] - base, r1 = ai[i + 1] - base;
    for (int k = r0; k < r1; k++)
      where[aj[k] - base] = k;
    for (int k = r0; k < diag[i]; k++) {
      const int c = aj[k] - base;
      S.uk.push_back(c);
      S.us.push_back(k);
      S.upiv.push_back(diag[c]);
      for (int m = diag[c] + 1; m < ai[c + 1] - base; m++) {
        const int w = where[aj[m] - base];
        if (w >= 0) {
          S.ptgt.push_back(w);
          S.psrc.push_back(m);
        }
      }
      S.pptr.push_back((int)S.ptgt.size());
    }
    for (int k = r0; k < r1; k++)
      where[aj[k] - base] = -1;
    S.uptr[i + 1] = (int)S.uk.size();
  }
}

} // namespace
} // namespace la

namespace la {
namespace {

__device__ __forceinline__ unsigned long long factor_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ int ld_acquire(const int *p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_release(int *p, int v) {
  asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// state[0]: chunk ticket, state[1]: a wait gave up, state[2]: smallest row
// whose pivot broke down (INT_MAX if none).
constexpr int kRowMax = 16;     // rows this long are worked on in shared memory
constexpr int kBatch = 4;       // updates whose index data and sources load together
constexpr int kBatchPairs = 12; // at most this many pairs in such a batch
// shared memory of the factor kernel: kRowMax values per thread, value-major
constexpr size_t kFactorSmem = sizeof(double) * kRowMax * kFactorThreads;

// The row being worked on: value q of this thread's row in shared memory,
// value-major so that a warp's accesses fall in distinct banks.
struct RowVals {
  double *base;
  __device__ double &operator[](int q) const { return base[q * kFactorThreads]; }
};

// Row j of at most kRowMax entries: its values live in shared memory (w)
// from the copy of vin to the final store.  The index data of
// a batch of updates (pair ranges, scalar and pivot indices, the pairs'
// target and source indices) does not depend on other rows, so the first
// batch's is loaded before the dependency wait; after it, the batch's source
// values are loaded together and the updates applied one after the other in
// their order -- the same exact operations in the same order as the general
// path, so the factor is unchanged.  A batch is cut short so that its pairs
// fit kBatchPairs; a single update with more pairs takes its pairs kGroup at
// a time.
template <int KIND>
__device__ void factor_short_row(const int j, const int rs, const int re,
                                 const int *__restrict__ uptr, const int *__restrict__ uk,
                                 const int *__restrict__ us, const int *__restrict__ upiv,
                                 const int *__restrict__ pptr, const int *__restrict__ ptgt,
                                 const int *__restrict__ psrc, const double *__restrict__ vin,
                                 double *v, const double diag_scale,
                                 const int *__restrict__ diag_of, int *done, int *state,
                                 const int sleep_ns) {
  const int len = re - rs;
  extern __shared__ double factor_smem[];
  const RowVals w{factor_smem + threadIdx.x};
  for (int q = 0; q < len; q++)
    w[q] = __ldg(vin + rs + q);
  if (KIND == kIC0)
    w[0] = __dmul_rn(w[0], diag_scale); // the (1 + omega) shift
  const int u0 = __ldg(uptr + j), u1 = __ldg(uptr + j + 1);
  int u = u0, nb = 0, np = 0;
  int e[kBatch + 1], sidx[kBatch], oidx[kBatch], tg[kBatchPairs], sr[kBatchPairs];
  auto load_batch = [&]() {
    nb = min(kBatch, u1 - u);
    for (int q = 0; q <= nb; q++)
      e[q] = __ldg(pptr + u + q);
    for (int q = 0; q < nb; q++) {
      sidx[q] = __ldg(KIND == kIC0 ? us + u + q : upiv + u + q);
      oidx[q] = KIND == kIC0 ? 0 : __ldg(us + u + q) - rs;
    }
    while (nb > 1 && e[nb] - e[0] > kBatchPairs)
      nb--;
    np = e[nb] - e[0];
    if (np <= kBatchPairs)
      for (int t = 0; t < np; t++) {
        tg[t] = __ldg(ptgt + e[0] + t) - rs;
        sr[t] = __ldg(psrc + e[0] + t);
      }
  };
  if (u < u1)
    load_batch();
  bool gave_up = false;
  const unsigned long long t0 = factor_ns();
  // every source row published: their flags polled kGroup at a time
  for (int g = u0; g < u1 && !gave_up; g += kGroup) {
    int kk[kGroup];
    unsigned pending = 0;
#pragma unroll
    for (int q = 0; q < kGroup; q++)
      if (g + q < u1) {
        kk[q] = __ldg(uk + g + q);
        pending |= 1u << q;
      }
    for (unsigned pass = 1; pending; pass++) {
      int f[kGroup];
#pragma unroll
      for (int q = 0; q < kGroup; q++)
        f[q] = (pending >> q) & 1u ? ld_acquire(done + kk[q]) : 1;
#pragma unroll
      for (int q = 0; q < kGroup; q++)
        if (f[q] != 0)
          pending &= ~(1u << q);
      if (pending && (pass & 63u) == 0u &&
          (ld_acquire(state + 1) != 0 || factor_ns() - t0 > kFactorWaitNs)) {
        atomicExch(state + 1, 1);
        gave_up = true;
        break;
      }
      if (pending && sleep_ns > 0) // back off: fewer polls crowding L2
        __nanosleep(sleep_ns);
    }
  }
  if (gave_up) // the row stays unpublished; the warp stops at its next claim
    return;
  while (u < u1) {
    double sv[kBatch];
    for (int q = 0; q < nb; q++)
      sv[q] = __ldcg(v + sidx[q]);
    if (np <= kBatchPairs) {
      double src[kBatchPairs];
      for (int t = 0; t < np; t++)
        src[t] = __ldcg(v + sr[t]);
      for (int q = 0; q < nb; q++) {
        double s;
        if (KIND == kIC0) {
          s = sv[q]; // U_kj, final
        } else {
          s = __ddiv_rn(w[oidx[q]], sv[q]); // L_jk = a_jk / u_kk
          w[oidx[q]] = s;
        }
        for (int t = e[q] - e[0]; t < e[q + 1] - e[0]; t++)
          w[tg[t]] = __dsub_rn(w[tg[t]], __dmul_rn(s, src[t]));
      }
    } else { // one update (nb == 1) with more pairs than a batch holds
      double s;
      if (KIND == kIC0) {
        s = sv[0];
      } else {
        s = __ddiv_rn(w[oidx[0]], sv[0]);
        w[oidx[0]] = s;
      }
      for (int eg = e[0]; eg < e[1]; eg += kGroup) {
        int tq[kGroup];
        double src[kGroup];
#pragma unroll
        for (int q = 0; q < kGroup; q++)
          if (eg + q < e[1]) {
            tq[q] = __ldg(ptgt + eg + q) - rs;
            src[q] = __ldcg(v + __ldg(psrc + eg + q));
          }
#pragma unroll
        for (int q = 0; q < kGroup; q++)
          if (eg + q < e[1])
            w[tq[q]] = __dsub_rn(w[tq[q]], __dmul_rn(s, src[q]));
      }
    }
    u += nb;
    if (u < u1)
      load_batch();
  }
  if (KIND == kIC0) {
    if (w[0] < 0.0)
      atomicMin(state + 2, j);
    const double piv = __dsqrt_rn(w[0]);
    w[0] = piv;
    for (int q = 1; q < len; q++)
      w[q] = __ddiv_rn(w[q], piv);
  } else if (w[__ldg(diag_of + j) - rs] == 0.0) {
    atomicMin(state + 2, j);
  }
  for (int q = 0; q < len; q++)
    v[rs + q] = w[q];
  __threadfence();
  st_release(done + j, 1);
}

// ---- One warp per row, for patterns whose rows receive many pairs (the
// 27-point stencils' ~90 a row): a lane per row would apply them one after
// another, each batch of indices and sources a dependent round trip.  Here
// the row's 32 lanes load its update indices, wait on its source rows, load
// up to kWarpPairs * 32 pairs' targets and source values together, then
// apply the updates one after another in their order, a lane per pair --
// an update's pairs have distinct targets, so each entry still sees exactly
// the host's operations in the host's order.  The row's values live in the
// warp's slice of shared memory (rows up to kWarpRowMax entries; longer
// ones are worked on in v, through L2).  Rows are claimed one at a time in
// level order from the ticket, so the lowest unfinished row always has its
// inputs and the pass cannot deadlock.
constexpr int kWarpRowMax = 128;
constexpr int kWarpPairs = 4;
constexpr size_t kWarpSmem = sizeof(double) * kWarpRowMax * (kFactorThreads / 32);

struct WarpRow {
  double *sh; // the warp's shared slice, or nullptr: the row's values in v
  double *g;  // v + rs
  __device__ double get(int q) const { return sh ? sh[q] : __ldcg(g + q); }
  __device__ void set(int q, double x) const {
    if (sh)
      sh[q] = x;
    else
      __stcg(g + q, x);
  }
};

template <int KIND>
__global__ void __launch_bounds__(kFactorThreads)
    factor_warp_kernel(const int n, const int *__restrict__ exec_row,
                       const int *__restrict__ rs_of, const int *__restrict__ diag_of,
                       const int *__restrict__ uptr, const int *__restrict__ uk,
                       const int *__restrict__ us, const int *__restrict__ upiv,
                       const int *__restrict__ pptr, const int *__restrict__ ptgt,
                       const int *__restrict__ psrc, const double *__restrict__ vin, double *v,
                       const double diag_scale, int *done, int *state, const int sleep_ns) {
  extern __shared__ double factor_smem[];
  const int lane = threadIdx.x & 31;
  double *slice = factor_smem + (threadIdx.x >> 5) * kWarpRowMax;
  for (;;) {
    int p = 0;
    if (lane == 0) // lane 0 alone decides; the warp leaves together
      p = ld_acquire(state + 1) != 0 ? n : atomicAdd(state, 1);
    p = __shfl_sync(0xffffffffu, p, 0);
    if (p >= n)
      return;
    const int j = __ldg(exec_row + p);
    const int rs = __ldg(rs_of + j), len = __ldg(rs_of + j + 1) - rs;
    const WarpRow w{len <= kWarpRowMax ? slice : nullptr, v + rs};
    for (int q = lane; q < len; q += 32)
      w.set(q, __ldg(vin + rs + q));
    __syncwarp();
    if (KIND == kIC0 && lane == 0)
      w.set(0, __dmul_rn(w.get(0), diag_scale)); // the (1 + omega) shift
    const int u0 = __ldg(uptr + j), u1 = __ldg(uptr + j + 1);
    // every source row published: a lane per update, polled together
    bool gave_up = false;
    const unsigned long long t0 = factor_ns();
    for (int ub = u0; ub < u1 && !gave_up; ub += 32) {
      const int k = ub + lane < u1 ? __ldg(uk + ub + lane) : -1;
      bool ready = k < 0;
      for (unsigned pass = 1;; pass++) {
        if (!ready)
          ready = ld_acquire(done + k) != 0;
        if (__all_sync(0xffffffffu, ready))
          break;
        if ((pass & 63u) == 0u) {
          bool stop = false;
          if (lane == 0)
            stop = ld_acquire(state + 1) != 0 || factor_ns() - t0 > kFactorWaitNs;
          if (__shfl_sync(0xffffffffu, stop, 0)) {
            gave_up = true;
            break;
          }
        }
        if (sleep_ns > 0)
          __nanosleep(sleep_ns);
      }
    }
    if (gave_up) { // the row stays unpublished; the warp stops at its next claim
      if (lane == 0)
        atomicExch(state + 1, 1);
      continue;
    }
    __syncwarp(); // the lanes' acquires order the source rows' values for all lanes
    for (int ub = u0; ub < u1; ub += 32) {
      const int nb = min(32, u1 - ub), u = ub + lane;
      int e0 = 0, e1 = 0, own = 0;
      double sv = 0.0;
      if (lane < nb) {
        e0 = __ldg(pptr + u);
        e1 = __ldg(pptr + u + 1);
        sv = __ldcg(v + __ldg(KIND == kIC0 ? us + u : upiv + u));
        if (KIND == kILU0)
          own = __ldg(us + u) - rs;
      }
      const int E0 = __shfl_sync(0xffffffffu, e0, 0), E1 = __shfl_sync(0xffffffffu, e1, nb - 1);
      const bool held = E1 - E0 <= 32 * kWarpPairs; // every pair in registers
      int tg[kWarpPairs];
      double src[kWarpPairs];
      if (held) {
#pragma unroll
        for (int r = 0; r < kWarpPairs; r++) {
          const int e = E0 + r * 32 + lane;
          tg[r] = e < E1 ? __ldg(ptgt + e) - rs : -1;
          src[r] = e < E1 ? __ldcg(v + __ldg(psrc + e)) : 0.0;
        }
      }
      for (int q = 0; q < nb; q++) {
        const int qe0 = __shfl_sync(0xffffffffu, e0, q), qe1 = __shfl_sync(0xffffffffu, e1, q);
        const double sq = __shfl_sync(0xffffffffu, sv, q);
        double s;
        if (KIND == kIC0) {
          s = sq; // U_kj, final
        } else {
          const int oq = __shfl_sync(0xffffffffu, own, q);
          s = __ddiv_rn(w.get(oq), sq); // L_jk = a_jk / u_kk
          __syncwarp();
          if (lane == 0)
            w.set(oq, s);
        }
        if (held) {
#pragma unroll
          for (int r = 0; r < kWarpPairs; r++) {
            const int e = E0 + r * 32 + lane;
            if (e >= qe0 && e < qe1)
              w.set(tg[r], __dsub_rn(w.get(tg[r]), __dmul_rn(s, src[r])));
          }
        } else {
          for (int e = qe0 + lane; e < qe1; e += 32) {
            const int t = __ldg(ptgt + e) - rs;
            w.set(t, __dsub_rn(w.get(t), __dmul_rn(s, __ldcg(v + __ldg(psrc + e)))));
          }
        }
        __syncwarp();
      }
    }
    if (KIND == kIC0) {
      double piv = 0.0;
      if (lane == 0) {
        const double d = w.get(0);
        if (d < 0.0)
          atomicMin(state + 2, j);
        piv = __dsqrt_rn(d);
        w.set(0, piv);
      }
      piv = __shfl_sync(0xffffffffu, piv, 0);
      for (int q = 1 + lane; q < len; q += 32)
        w.set(q, __ddiv_rn(w.get(q), piv));
    } else if (lane == 0 && w.get(__ldg(diag_of + j) - rs) == 0.0) {
      atomicMin(state + 2, j);
    }
    __syncwarp();
    if (w.sh)
      for (int q = lane; q < len; q += 32)
        v[rs + q] = w.sh[q];
    __syncwarp();
    if (lane == 0) {
      __threadfence();
      st_release(done + j, 1);
    }
  }
}

template <int KIND>
__global__ void __launch_bounds__(kFactorThreads)
    factor_kernel(const int nchunks, const int *__restrict__ chunk_start,
                  const int *__restrict__ exec_row, const int *__restrict__ rs_of,
                  const int *__restrict__ diag_of, const int *__restrict__ uptr,
                  const int *__restrict__ uk, const int *__restrict__ us,
                  const int *__restrict__ upiv, const int *__restrict__ pptr,
                  const int *__restrict__ ptgt, const int *__restrict__ psrc,
                  const double *__restrict__ vin, double *v, const double diag_scale, int *done,
                  int *state, const int sleep_ns) {
  const int lane = threadIdx.x & 31;
  for (;;) {
    // lane 0 alone decides (a wait gave up somewhere: stop) and broadcasts,
    // so the whole warp leaves together; no lane ever returns on its own
    int c = 0;
    if (lane == 0)
      c = ld_acquire(state + 1) != 0 ? nchunks : atomicAdd(state, 1);
    c = __shfl_sync(0xffffffffu, c, 0);
    if (c >= nchunks)
      return;
    const int p = __ldg(chunk_start + c) + lane;
    if (p >= __ldg(chunk_start + c + 1))
      continue;
    const int j = __ldg(exec_row + p);
    const int rs = __ldg(rs_of + j), re = __ldg(rs_of + j + 1);
    if (re - rs <= kRowMax) {
      factor_short_row<KIND>(j, rs, re, uptr, uk, us, upiv, pptr, ptgt, psrc, vin, v, diag_scale,
                             diag_of, done, state, sleep_ns);
      continue;
    }
    for (int q = rs; q < re; q++)
      v[q] = __ldg(vin + q);
    if (KIND == kIC0)
      v[rs] = __dmul_rn(__ldg(vin + rs), diag_scale); // the (1 + omega) shift
    bool gave_up = false;
    const int u0 = __ldg(uptr + j), u1 = __ldg(uptr + j + 1);
    const unsigned long long t0 = factor_ns();
    // every source row published: their flags polled kGroup at a time
    for (int g = u0; g < u1 && !gave_up; g += kGroup) {
      int kk[kGroup];
      unsigned pending = 0;
#pragma unroll
      for (int q = 0; q < kGroup; q++)
        if (g + q < u1) {
          kk[q] = __ldg(uk + g + q);
          pending |= 1u << q;
        }
      for (unsigned pass = 1; pending; pass++) {
        int f[kGroup];
#pragma unroll
        for (int q = 0; q < kGroup; q++)
          f[q] = (pending >> q) & 1u ? ld_acquire(done + kk[q]) : 1;
#pragma unroll
        for (int q = 0; q < kGroup; q++)
          if (f[q] != 0)
            pending &= ~(1u << q);
        if (pending && (pass & 63u) == 0u &&
            (ld_acquire(state + 1) != 0 || factor_ns() - t0 > kFactorWaitNs)) {
          atomicExch(state + 1, 1);
          gave_up = true;
          break;
        }
        if (pending && sleep_ns > 0)
          __nanosleep(sleep_ns);
      }
    }
    // the updates in their order; an update's scalar operand and its pairs'
    // sources (final values of its source row) are loaded together, kGroup
    // pairs at a time, then applied in order -- the same operations in the
    // same order as one at a time
    for (int u = u0; u < u1 && !gave_up; u++) {
      const int e0 = __ldg(pptr + u), e1 = __ldg(pptr + u + 1);
      const double sv = __ldcg(v + __ldg(KIND == kIC0 ? us + u : upiv + u));
      double s = 0.0;
      for (int eg = e0; eg == e0 || eg < e1; eg += kGroup) {
        int tg[kGroup];
        double src[kGroup];
#pragma unroll
        for (int q = 0; q < kGroup; q++)
          if (eg + q < e1) {
            tg[q] = __ldg(ptgt + eg + q);
            src[q] = __ldcg(v + __ldg(psrc + eg + q));
          }
        if (eg == e0) {
          if (KIND == kIC0) {
            s = sv; // U_kj, final
          } else {
            const int own = __ldg(us + u); // L_jk = a_jk / u_kk
            s = __ddiv_rn(v[own], sv);
            v[own] = s;
          }
        }
#pragma unroll
        for (int q = 0; q < kGroup; q++)
          if (eg + q < e1)
            v[tg[q]] = __dsub_rn(v[tg[q]], __dmul_rn(s, src[q]));
        if (eg + kGroup >= e1)
          break;
      }
    }
    if (gave_up) // the row stays unpublished; the warp stops at its next claim
      continue;
    if (KIND == kIC0) {
      if (v[rs] < 0.0)
        atomicMin(state + 2, j);
      const double piv = __dsqrt_rn(v[rs]);
      v[rs] = piv;
      for (int q = rs + 1; q < re; q++)
        v[q] = __ddiv_rn(v[q], piv);
    } else if (v[__ldg(diag_of + j)] == 0.0) {
      atomicMin(state + 2, j);
    }
    __threadfence();
    st_release(done + j, 1);
  }
}

// level of every row (longest path over its updates' source rows, which all
// precede it), rows sorted by (level, row), 32-row chunks inside levels
void schedule(int n, const Symbolic &S, std::vector<int> &erow, std::vector<int> &cstart,
              int *levels) {
  std::vector<int> lvl(n, 0);
  int top = 0;
  for (int j = 0; j < n; j++) {
    int l = 0;
    for (int u = S.uptr[j]; u < S.uptr[j + 1]; u++)
      l = std::max(l, lvl[S.uk[u]] + 1);
    lvl[j] = l;
    top = std::max(top, l + 1);
  }
  *levels = n ? top : 0;
  std::vector<int> start(top + 1, 0);
  for (int j = 0; j < n; j++)
    start[lvl[j] + 1]++;
  for (int l = 0; l < top; l++)
    start[l + 1] += start[l];
  erow.resize(n);
  std::vector<int> fill(start.begin(), start.end() - 1);
  for (int j = 0; j < n; j++)
    erow[fill[lvl[j]]++] = j;
  cstart.clear();
  for (int l = 0; l < top; l++)
    for (int p = start[l]; p < start[l + 1]; p += kFactorChunk)
      cstart.push_back(p);
  cstart.push_back(n);
}

la_status plan_finish(la_factor_plan_s *P);

la_status plan_build(la_factor_plan_s *P, const int *ai, const int *aj, Symbolic &S) {
  const int n = P->n;
  std::vector<int> erow, cstart;
  schedule(n, S, erow, cstart, &P->levels);
  P->nchunks = (int)cstart.size() - 1;
  P->npairs = (long long)S.ptgt.size();
  std::vector<int> rs(n + 1);
  for (int j = 0; j <= n; j++)
    rs[j] = ai[j] - P->base;
  auto up = [](DevBuf &b, const std::vector<int> &v) {
    return b.upload(v.empty() ? nullptr : v.data(), sizeof(int) * std::max<size_t>(v.size(), 1));
  };
  // empty lists still get a (1-entry) buffer so every pointer is valid
  for (std::vector<int> *v : {&S.uk, &S.us, &S.upiv, &S.ptgt, &S.psrc})
    if (v->empty())
      v->push_back(0);
  LA_TRY(up(P->rs, rs));
  LA_TRY(up(P->diag, S.diag.empty() ? std::vector<int>{0} : S.diag));
  LA_TRY(up(P->exec_row, erow.empty() ? std::vector<int>{0} : erow));
  LA_TRY(up(P->chunk_start, cstart));
  LA_TRY(up(P->uptr, S.uptr));
  LA_TRY(up(P->uk, S.uk));
  LA_TRY(up(P->us, S.us));
  LA_TRY(up(P->upiv, S.upiv));
  LA_TRY(up(P->pptr, S.pptr));
  LA_TRY(up(P->ptgt, S.ptgt));
  LA_TRY(up(P->psrc, S.psrc));
  return plan_finish(P);
}

// The numeric pass's work buffers and grid (either plan builder).
la_status plan_finish(la_factor_plan_s *P) {
  const int n = P->n;
  LA_TRY(P->vin.alloc(sizeof(double) * std::max(P->nnz, 1)));
  LA_TRY(P->done.alloc(sizeof(int) * std::max(n, 1)));
  LA_TRY(P->state.alloc(sizeof(int) * 4));
  // one warp per row when rows receive many pairs (more than 8 on average);
  // LA_FACTOR_WARP=0/1 forces either form (testing / tuning override)
  P->warp = P->npairs > 8LL * n;
  if (const char *e = std::getenv("LA_FACTOR_WARP"))
    P->warp = std::atoi(e) != 0;
  int per_sm = 0;
  if (P->warp)
    LA_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, (const void *)factor_warp_kernel<kIC0>, kFactorThreads, kWarpSmem));
  else
    LA_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, (const void *)factor_kernel<kIC0>, kFactorThreads, kFactorSmem));
  // LA_FACTOR_CTAS_PER_SM caps the CTAs per SM (tuning override; default:
  // as many as fit).  Warps beyond what the widest levels use only poll.
  per_sm = std::max(per_sm, 1);
  P->sleep_ns = kPollSleepNs;
  if (const char *e = std::getenv("LA_FACTOR_SLEEP_NS")) // tuning override
    P->sleep_ns = std::max(0, std::atoi(e));
  if (const char *e = std::getenv("LA_FACTOR_CTAS_PER_SM"))
    per_sm = std::min(per_sm, std::max(1, std::atoi(e)));
  const int units = P->warp ? n : P->nchunks; // what a warp claims: a row or a chunk
  const int need = (units + kFactorThreads / 32 - 1) / (kFactorThreads / 32);
  P->grid = std::max(1, std::min(per_sm * sm_count(), need));
  return LA_OK;
}

// ---- The IC(0) plan built on the device (large patterns).  The same
// lists as symbolic_ic0 + schedule, step for step: each row's updates are
// the strict upper entries of its column (counted, placed in any order,
// then insertion-sorted per row by update_before), the pairs are counted,
// scanned and written per update, the levels come from the depth solve
// over the updates, and the rows are sorted by (level, row) with 32-row
// chunks inside levels.  Integer work only: the plan equals the host's.

constexpr int kDevicePlanRows = 65536; // smaller patterns: the host's plan
constexpr int kDeviceSortMax = 512;    // a longer update list: the host's plan

int plan_grid(int n) { return std::max(1, std::min((n + 255) / 256, 8 * sm_count())); }

__global__ void sym_rebase_kernel(const int m, const int base, int *v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
    v[i] -= base;
}

// cnt[c] = strict upper entries in column c
__global__ void sym_col_count_kernel(const int n, const int *__restrict__ ai,
                                     const int *__restrict__ aj, int *cnt) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
    for (int e = ai[k] + 1; e < ai[k + 1]; e++)
      atomicAdd(cnt + aj[e], 1);
}

// each strict upper entry e = (k, c) becomes an update of row c (any order)
__global__ void sym_col_fill_kernel(const int n, const int *__restrict__ ai,
                                    const int *__restrict__ aj, int *cursor, int *uk, int *us) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
    for (int e = ai[k] + 1; e < ai[k + 1]; e++) {
      const int q = atomicAdd(cursor + aj[e], 1);
      uk[q] = k;
      us[q] = e;
    }
}

// update_before on the device (the same rule)
__device__ bool update_before_dev(const int *__restrict__ aj, int px, int lx, int py, int ly) {
  for (bool flip = false;; flip = !flip) {
    const int cx = __ldg(aj + px), cy = __ldg(aj + py);
    if (cx != cy)
      return (cx > cy) != flip;
    if (px == lx)
      return !flip;
    if (py == ly)
      return flip;
    px--;
    py--;
  }
}

// row j's updates sorted in place (insertion sort on its own slice)
__global__ void sym_order_kernel(const int n, const int *__restrict__ ai,
                                 const int *__restrict__ aj, const int *__restrict__ uptr,
                                 int *uk, int *us, int *too_long) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const int u0 = uptr[j], u1 = uptr[j + 1];
    if (u1 - u0 > kDeviceSortMax) {
      atomicExch(too_long, 1);
      continue;
    }
    for (int u = u0 + 1; u < u1; u++) {
      const int e = us[u], k = uk[u], lk = ai[k];
      int w = u;
      while (w > u0) {
        const int e2 = us[w - 1], k2 = uk[w - 1];
        if (!update_before_dev(aj, e - 1, lk, e2 - 1, ai[k2]))
          break;
        us[w] = e2;
        uk[w] = k2;
        w--;
      }
      us[w] = e;
      uk[w] = k;
    }
  }
}

// the pairs of update u of row j: columns of row k from entry us[u] on that
// row j holds (visit(u, p, ck) per pair, ascending)
template <typename F>
__device__ void sym_pairs(const int *__restrict__ ai, const int *__restrict__ aj, int j, int k,
                          int ck0, F visit) {
  const int re = ai[j + 1], ke = ai[k + 1];
  for (int p = ai[j], ck = ck0; ck < ke && p < re;) {
    const int a = __ldg(aj + ck), b = __ldg(aj + p);
    if (a == b)
      visit(p++, ck++);
    else if (a < b)
      ck++;
    else
      p++;
  }
}

__global__ void sym_pair_count_kernel(const int n, const int *__restrict__ ai,
                                      const int *__restrict__ aj, const int *__restrict__ uptr,
                                      const int *__restrict__ uk, const int *__restrict__ us,
                                      int *pcount) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
    for (int u = uptr[j]; u < uptr[j + 1]; u++) {
      int c = 0;
      sym_pairs(ai, aj, j, uk[u], us[u], [&](int, int) { c++; });
      pcount[u] = c;
    }
}

__global__ void sym_pair_fill_kernel(const int n, const int *__restrict__ ai,
                                     const int *__restrict__ aj, const int *__restrict__ uptr,
                                     const int *__restrict__ uk, const int *__restrict__ us,
                                     const int *__restrict__ pptr, int *ptgt, int *psrc) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
    for (int u = uptr[j]; u < uptr[j + 1]; u++) {
      int w = pptr[u];
      sym_pairs(ai, aj, j, uk[u], us[u], [&](int p, int ck) {
        ptgt[w] = p;
        psrc[w++] = ck;
      });
    }
}

// flag[p] = 1 where a 32-row chunk starts (level start, then every 32 rows)
__global__ void chunk_flag_kernel(const int n, const unsigned *__restrict__ level,
                                  const int *__restrict__ starts, int *flag) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p <= n; p += gridDim.x * blockDim.x)
    flag[p] = p < n && ((p - starts[level[p]]) & (kFactorChunk - 1)) == 0;
}

__global__ void chunk_scatter_kernel(const int n, const unsigned *__restrict__ level,
                                     const int *__restrict__ starts, const int *__restrict__ pos,
                                     int *chunk_start) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p <= n; p += gridDim.x * blockDim.x)
    if (p == n)
      chunk_start[pos[n]] = n;
    else if (((p - starts[level[p]]) & (kFactorChunk - 1)) == 0)
      chunk_start[pos[p]] = p;
}

void take(DevBuf &dst, DevBuf &src) {
  std::swap(dst.p, src.p);
  std::swap(dst.bytes, src.bytes);
}

// *ok = false (nothing built): a row receives more than kDeviceSortMax
// updates; the caller builds the host's plan instead.
la_status plan_build_ic0_device(la_factor_plan_s *P, const int *ai, const int *aj, bool *ok) {
  *ok = false;
  const int n = P->n, nnz = P->nnz, base = P->base;
  cudaStream_t st = nullptr;
  const int g = plan_grid(n);
  DevBuf dai, daj, uptr, cursor, uk, us, flag, pptr, ptgt, psrc;
  LA_TRY(dai.upload(ai, sizeof(int) * (n + 1)));
  LA_TRY(daj.upload(aj, sizeof(int) * std::max(nnz, 1)));
  sym_rebase_kernel<<<g, 256, 0, st>>>(n + 1, base, dai.as<int>());
  sym_rebase_kernel<<<plan_grid(nnz), 256, 0, st>>>(nnz, base, daj.as<int>());
  LA_TRY(uptr.alloc(sizeof(int) * (n + 1)));
  LA_CUDA_TRY(cudaMemsetAsync(uptr.p, 0, sizeof(int) * (n + 1), st));
  sym_col_count_kernel<<<g, 256, 0, st>>>(n, dai.as<int>(), daj.as<int>(), uptr.as<int>());
  LA_CUDA_TRY(cudaGetLastError());
  LA_TRY(scan_exclusive(uptr.as<int>(), n + 1, st));
  int nu = 0;
  LA_CUDA_TRY(cudaMemcpyAsync(&nu, uptr.as<int>() + n, sizeof(int), cudaMemcpyDeviceToHost, st));
  LA_CUDA_TRY(cudaStreamSynchronize(st));
  LA_TRY(uk.alloc(sizeof(int) * std::max(nu, 1)));
  LA_TRY(us.alloc(sizeof(int) * std::max(nu, 1)));
  LA_TRY(cursor.alloc(sizeof(int) * (n + 1)));
  LA_CUDA_TRY(cudaMemcpyAsync(cursor.p, uptr.p, sizeof(int) * (n + 1), cudaMemcpyDeviceToDevice,
                              st));
  sym_col_fill_kernel<<<g, 256, 0, st>>>(n, dai.as<int>(), daj.as<int>(), cursor.as<int>(),
                                         uk.as<int>(), us.as<int>());
  LA_CUDA_TRY(cudaMemsetAsync(cursor.p, 0, sizeof(int), st)); // the too-long flag
  sym_order_kernel<<<g, 256, 0, st>>>(n, dai.as<int>(), daj.as<int>(), uptr.as<int>(),
                                      uk.as<int>(), us.as<int>(), cursor.as<int>());
  LA_CUDA_TRY(cudaGetLastError());
  int too_long = 0;
  LA_CUDA_TRY(cudaMemcpyAsync(&too_long, cursor.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  LA_CUDA_TRY(cudaStreamSynchronize(st));
  if (too_long)
    return LA_OK;
  LA_TRY(pptr.alloc(sizeof(int) * ((size_t)nu + 1)));
  LA_CUDA_TRY(cudaMemsetAsync(pptr.as<int>() + nu, 0, sizeof(int), st));
  sym_pair_count_kernel<<<g, 256, 0, st>>>(n, dai.as<int>(), daj.as<int>(), uptr.as<int>(),
                                           uk.as<int>(), us.as<int>(), pptr.as<int>());
  LA_CUDA_TRY(cudaGetLastError());
  LA_TRY(scan_exclusive(pptr.as<int>(), nu + 1, st));
  int npairs = 0;
  LA_CUDA_TRY(cudaMemcpyAsync(&npairs, pptr.as<int>() + nu, sizeof(int), cudaMemcpyDeviceToHost,
                              st));
  LA_CUDA_TRY(cudaStreamSynchronize(st));
  LA_TRY(ptgt.alloc(sizeof(int) * std::max(npairs, 1)));
  LA_TRY(psrc.alloc(sizeof(int) * std::max(npairs, 1)));
  sym_pair_fill_kernel<<<g, 256, 0, st>>>(n, dai.as<int>(), daj.as<int>(), uptr.as<int>(),
                                          uk.as<int>(), us.as<int>(), pptr.as<int>(),
                                          ptgt.as<int>(), psrc.as<int>());
  LA_CUDA_TRY(cudaGetLastError());
  // levels: row j depends on the rows of its updates, all earlier rows
  DevBuf order, keys, starts;
  int lv = 0;
  LA_TRY(levels_on_device(LA_LOWER, n, 0, uptr.as<int>(), uk.as<int>(), order, keys, starts, &lv,
                          st));
  LA_TRY(flag.alloc(sizeof(int) * (n + 1)));
  chunk_flag_kernel<<<g, 256, 0, st>>>(n, keys.as<unsigned>(), starts.as<int>(), flag.as<int>());
  LA_CUDA_TRY(cudaGetLastError());
  LA_TRY(scan_exclusive(flag.as<int>(), n + 1, st));
  int nchunks = 0;
  LA_CUDA_TRY(cudaMemcpyAsync(&nchunks, flag.as<int>() + n, sizeof(int), cudaMemcpyDeviceToHost,
                              st));
  LA_CUDA_TRY(cudaStreamSynchronize(st));
  LA_TRY(P->chunk_start.alloc(sizeof(int) * (nchunks + 1)));
  chunk_scatter_kernel<<<g, 256, 0, st>>>(n, keys.as<unsigned>(), starts.as<int>(),
                                          flag.as<int>(), P->chunk_start.as<int>());
  LA_CUDA_TRY(cudaGetLastError());
  LA_TRY(P->diag.alloc(sizeof(int) * n));
  LA_CUDA_TRY(cudaMemcpyAsync(P->diag.p, dai.p, sizeof(int) * n, cudaMemcpyDeviceToDevice, st));
  LA_TRY(P->upiv.alloc(sizeof(int)));
  LA_CUDA_TRY(cudaMemsetAsync(P->upiv.p, 0, sizeof(int), st));
  LA_CUDA_TRY(cudaStreamSynchronize(st));
  take(P->rs, dai);
  take(P->exec_row, order);
  take(P->uptr, uptr);
  take(P->uk, uk);
  take(P->us, us);
  take(P->pptr, pptr);
  take(P->ptgt, ptgt);
  take(P->psrc, psrc);
  P->levels = lv;
  P->nchunks = nchunks;
  P->npairs = npairs;
  LA_TRY(plan_finish(P));
  *ok = true;
  return LA_OK;
}

} // namespace

// Values in (host or device), factor out (host or device), on `st`;
// synchronises st.  *bad_row: the smallest row that broke down, or -1.
la_status factor_numeric(la_factor_plan_s *P, const double *av, double omega, double *out,
                         bool on_device, int *bad_row, cudaStream_t st) {
  *bad_row = -1;
  if (P->n == 0)
    return LA_OK;
  const size_t bytes = sizeof(double) * P->nnz;
  DevBuf tmp;
  double *v = out;
  if (!on_device) {
    LA_TRY(tmp.alloc(std::max<size_t>(bytes, 8)));
    v = tmp.as<double>();
  }
  if (bytes)
    LA_CUDA_TRY(cudaMemcpyAsync(P->vin.p, av, bytes,
                                on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                st));
  const int init[4] = {0, 0, 0x7fffffff, 0};
  LA_CUDA_TRY(cudaMemcpyAsync(P->state.p, init, sizeof(init), cudaMemcpyHostToDevice, st));
  LA_CUDA_TRY(cudaMemsetAsync(P->done.p, 0, sizeof(int) * P->n, st));
  if (P->warp) {
    auto launch = P->kind == kIC0 ? factor_warp_kernel<kIC0> : factor_warp_kernel<kILU0>;
    launch<<<P->grid, kFactorThreads, kWarpSmem, st>>>(
        P->n, P->exec_row.as<int>(), P->rs.as<int>(), P->diag.as<int>(), P->uptr.as<int>(),
        P->uk.as<int>(), P->us.as<int>(), P->upiv.as<int>(), P->pptr.as<int>(),
        P->ptgt.as<int>(), P->psrc.as<int>(), P->vin.as<double>(), v, 1.0 + omega,
        P->done.as<int>(), P->state.as<int>(), P->sleep_ns);
  } else {
    auto launch = P->kind == kIC0 ? factor_kernel<kIC0> : factor_kernel<kILU0>;
    launch<<<P->grid, kFactorThreads, kFactorSmem, st>>>(
        P->nchunks, P->chunk_start.as<int>(), P->exec_row.as<int>(), P->rs.as<int>(),
        P->diag.as<int>(), P->uptr.as<int>(), P->uk.as<int>(), P->us.as<int>(),
        P->upiv.as<int>(), P->pptr.as<int>(), P->ptgt.as<int>(), P->psrc.as<int>(),
        P->vin.as<double>(), v, 1.0 + omega, P->done.as<int>(), P->state.as<int>(),
        P->sleep_ns);
  }
  LA_CUDA_TRY(cudaGetLastError());
  int state[4];
  LA_CUDA_TRY(cudaMemcpyAsync(state, P->state.p, sizeof(state), cudaMemcpyDeviceToHost, st));
  if (!on_device && bytes)
    LA_CUDA_TRY(cudaMemcpyAsync(out, v, bytes, cudaMemcpyDeviceToHost, st));
  LA_CUDA_TRY(cudaStreamSynchronize(st));
  if (state[1]) {
    set_error("numeric factorisation: a dependency wait exceeded its 1 s bound");
    return LA_ERR_TIMEOUT;
  }
  if (state[2] != 0x7fffffff) {
    *bad_row = state[2];
    set_error(P->kind == kIC0 ? "IC(0) breakdown: negative pivot in row %d (omega = %g)"
                              : "ILU(0): zero pivot in row %d",
              state[2], omega);
    return LA_ERR_BREAKDOWN;
  }
  return LA_OK;
}

la_status factor_plan_create(int kind, int n, int base, const int *ai, const int *aj,
                             la_factor_plan_t *out) {
  std::unique_ptr<la_factor_plan_s> P(new la_factor_plan_s());
  P->kind = kind;
  P->n = n;
  P->base = base;
  P->nnz = ai[n] - base;
  P->h_ai.assign(ai, ai + n + 1);
  if (kind == kIC0 && n >= kDevicePlanRows) {
    bool ok = false;
    LA_TRY(plan_build_ic0_device(P.get(), ai, aj, &ok));
    if (ok) {
      *out = P.release();
      return LA_OK;
    }
  }
  Symbolic S;
  if (kind == kIC0) {
    symbolic_ic0(n, base, ai, aj, S);
  } else {
    std::vector<int> diag(n);
    for (int i = 0; i < n; i++) {
      const int *lo = aj + ai[i] - base, *hi = aj + ai[i + 1] - base;
      const int *at = std::lower_bound(lo, hi, i + base);
      if (at == hi || *at != i + base) {
        set_error("ILU(0): row %d has no diagonal entry", i);
        return LA_ERR_INVALID_ARG;
      }
      diag[i] = (int)(at - aj);
    }
    symbolic_ilu0(n, base, ai, aj, diag, S);
  }
  if (n)
    LA_TRY(plan_build(P.get(), ai, aj, S));
  *out = P.release();
  return LA_OK;
}

} // namespace la
