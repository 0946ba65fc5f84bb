// la_trsv.cu -- level-scheduled sparse triangular solve, one kernel launch
// per solve.
//
// Reference: OptimizedTriangularSolve<Barrier, L|U> (sparse_mat_op/
// triangle_solve.hpp:149-208, triangle_solve.tpp:17-155).  analysis()
// computes level sets with TopologicalSort2 (matrix_utils.hpp:637-675),
// splits every level over the threads and stores the rows physically in
// execution order (permuteRow); the apply walks the levels with an OpenMP
// barrier after each one and computes
//   x[i] = diag ? (b[i] - sum_j T_ij x[j]) / diag[i] : b[i] - sum_j T_ij x[j].
//
// B200 design.  The same host analysis (bit-identical level sets) feeds one
// of two schedules, both computing every x_i with the reference's exact
// operations in stored column order (so the results are bit-identical):
//
// Level order (schedule 0).  Rows are stored in level order and cut into
// 32-row chunks that never straddle a level.  One launch of a persistent
// grid walks all levels: warps claim chunks in order from an atomic ticket,
// one lane per row.  Instead of a grid barrier per level, each lane waits
// only for the x entries its row reads: x is pre-filled with a sentinel NaN
// bit pattern and a finished row publishes x[i] with a device-scope store,
// so a dependency is ready when its x entry stops being the sentinel (the
// value is its own flag; one L2 round trip).  Because chunks are claimed in
// level order, the lowest unfinished chunk always has its inputs ready and
// the solve cannot deadlock.
//
// Partitioned (schedule 1).  The rows are split into parts whose dependency
// graph is acyclic and shallow (la_partition.cpp), one co-resident CTA per
// part (cooperative launch).  A CTA walks the levels present in its part with
// one __syncthreads per level and keeps its rows' x values in shared memory,
// so a dependency inside the part is a shared-memory read; a dependency on
// another part is awaited in global memory as above.  A dependency path
// crosses few part boundaries, so most of the per-level cost is a
// shared-memory step instead of an L2 round trip.  No deadlock: every CTA is
// resident and processes its rows in level order, so the unfinished row of
// lowest level always has its inputs ready.  The analysis models both
// schedules' critical paths and keeps the partitioned one when it is clearly
// shorter.
//
// Every wait is bounded by the global timer; on expiry the kernel records a
// timeout in the plan's error word and all warps leave.
//
// Roofline: latency-bound at these sizes (levels x per-level step); the
// algorithmic bytes per solve are
//   nnz*(sizeof(V)+4) + (n+1)*4 + n*4 [exec->row map] + n*sizeof(V) [diag]
//   + n*sizeof(X) [b] + n*sizeof(X) [x].

#include "la_device.cuh"
#include "la_internal.h"

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <numeric>
#include <vector>

namespace la {
namespace {

constexpr int kThreads = 256;
constexpr int kChunk = 32;
constexpr int kDeps = 8; // dependency loads issued together per row
constexpr unsigned long long kWaitNs = 1000000000ull; // 1 s per wait
constexpr int kDeviceLevelsRows = 65536; // level sets on the GPU from this size

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

template <typename X> struct Sentinel;
template <> struct Sentinel<double> {
  static constexpr unsigned long long bits = 0xffffffffffffffffull;
  static __device__ __forceinline__ bool is(double v) {
    return (unsigned long long)__double_as_longlong(v) == bits;
  }
  static __device__ __forceinline__ double scrub(double v) {
    return is(v) ? __longlong_as_double(0x7ff8000000000000ll) : v;
  }
};
template <> struct Sentinel<float> {
  static constexpr unsigned bits = 0xffffffffu;
  static __device__ __forceinline__ bool is(float v) {
    return (unsigned)__float_as_uint(v) == bits;
  }
  static __device__ __forceinline__ float scrub(float v) {
    return is(v) ? __uint_as_float(0x7fc00000u) : v;
  }
};

__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double div_rn(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float div_rn(float a, float b) { return __fdiv_rn(a, b); }

// Warps claim 32-row chunks in level order from an atomic ticket, one lane
// per row.  A chunk is claimed only after every earlier chunk has been
// claimed by a running warp, so the lowest unfinished chunk always has its
// inputs ready and the solve cannot deadlock, whatever the grid size.
//
// Each lane runs its row as a small state machine inside a warp-uniform
// loop, so a row is published the moment its own inputs are present rather
// than when the slowest lane of the warp is done: dependencies are read
// kDeps at a time (all loads issued before any is checked, so a level costs
// one L2 round trip), still-missing ones are re-polled each pass, and the
// sum is formed in stored column order with exact (never fused) operations,
// so each x_i is bit-identical to the reference's
//   x[idx] = diag ? (b[idx] - val) / diag[idx] : b[idx] - val.
template <typename V, typename X, bool UNIT>
__global__ void __launch_bounds__(kThreads)
    trsv_level_kernel_grouped(const int nchunks, const int *__restrict__ chunk_start,
                      const int *__restrict__ ai, const int *__restrict__ aj,
                      const V *__restrict__ av, const V *__restrict__ diag,
                      const int *__restrict__ exec_row,
                      const X *__restrict__ b, X *x, const int base, int *err,
                      int *ticket) {
  const int lane = threadIdx.x & 31;
  for (;;) {
    int c = 0;
    if (lane == 0)
      c = atomicAdd(ticket, 1);
    c = __shfl_sync(0xffffffffu, c, 0);
    if (c >= nchunks)
      return;
    const int p = __ldg(chunk_start + c) + lane;
    bool done = p >= __ldg(chunk_start + c + 1);
    int i = 0, k0 = 0, ke = 0;
    unsigned pend = 0;
    int jj[kDeps];
    X a[kDeps], xv[kDeps];
    X sum = X(0);
    // load the dependency group starting at k0; returns the missing mask
    auto load_group = [&]() {
      unsigned m = 0;
#pragma unroll
      for (int q = 0; q < kDeps; q++)
        if (k0 + q < ke) {
          jj[q] = __ldg(aj + k0 + q) - base;
          a[q] = X(__ldg(av + k0 + q));
        }
#pragma unroll
      for (int q = 0; q < kDeps; q++)
        if (k0 + q < ke) {
          xv[q] = dev::ld_relaxed(x + jj[q]);
          if (Sentinel<X>::is(xv[q]))
            m |= 1u << q;
        }
      return m;
    };
    if (!done) {
      i = __ldg(exec_row + p);
      k0 = __ldg(ai + p) - base;
      ke = __ldg(ai + p + 1) - base;
      pend = load_group();
    }
    const unsigned long long t0 = global_ns();
    for (unsigned pass = 1;; pass++) {
      if (!done) {
        if (pend) {
#pragma unroll
          for (int q = 0; q < kDeps; q++)
            if (pend & (1u << q)) {
              xv[q] = dev::ld_relaxed(x + jj[q]);
              if (!Sentinel<X>::is(xv[q]))
                pend &= ~(1u << q);
            }
        }
        if (!pend) {
#pragma unroll
          for (int q = 0; q < kDeps; q++)
            if (k0 + q < ke)
              sum = add_rn(sum, mul_rn(a[q], xv[q]));
          k0 += kDeps;
          if (k0 < ke) {
            pend = load_group();
          } else {
            X xi = sub_rn(__ldg(b + i), sum);
            if (!UNIT)
              xi = div_rn(xi, X(__ldg(diag + p)));
            dev::st_relaxed(x + i, Sentinel<X>::scrub(xi));
            done = true;
          }
        }
      }
      if (__all_sync(0xffffffffu, done))
        break;
      bool abort = false;
      if ((pass & 31u) == 0u && lane == 0)
        abort = dev::ld_relaxed(err) != 0 || global_ns() - t0 > kWaitNs;
      if (__shfl_sync(0xffffffffu, abort, 0)) {
        if (lane == 0)
          atomicExch(err, 1);
        return;
      }
      if (!done && pend)
        __nanosleep(32);
    }
  }
}

// Rows with at most KD stored entries (the plan picks the smallest KD in
// {4, 8, 16} that covers its longest row): the same state machine with one
// dependency group kept entirely in registers and no sleep between polls --
// measured on the RCM-ordered 128^3 IC(0) factor, the shorter pass this gives
// cuts the cost of a level from 2.4 us (grouped form) to about 1.6 us.
template <typename V, typename X, bool UNIT, int KD>
__global__ void __launch_bounds__(kThreads)
    trsv_level_kernel(const int nchunks, const int *__restrict__ chunk_start,
                      const int *__restrict__ ai, const int *__restrict__ aj,
                      const V *__restrict__ av, const V *__restrict__ diag,
                      const int *__restrict__ exec_row,
                      const X *__restrict__ b, X *x, const int base, int *err,
                      int *ticket, const int sleep_ns) {
  const int lane = threadIdx.x & 31;
  for (;;) {
    int c = 0;
    if (lane == 0)
      c = atomicAdd(ticket, 1);
    c = __shfl_sync(0xffffffffu, c, 0);
    if (c >= nchunks)
      return;
    const int p = __ldg(chunk_start + c) + lane;
    bool done = p >= __ldg(chunk_start + c + 1);
    int i = 0, kb = 0, ke = 0;
    int jj[KD];
    X a[KD], xv[KD];
    unsigned pend = 0;
    if (!done) {
      i = __ldg(exec_row + p);
      kb = __ldg(ai + p) - base;
      ke = __ldg(ai + p + 1) - base;
#pragma unroll
      for (int q = 0; q < KD; q++)
        if (kb + q < ke) {
          jj[q] = __ldg(aj + kb + q) - base;
          a[q] = X(__ldg(av + kb + q));
          pend |= 1u << q;
        }
    }
    const unsigned long long t0 = global_ns();
    for (unsigned pass = 1;; pass++) {
      if (!done) {
#pragma unroll
        for (int q = 0; q < KD; q++)
          if (pend & (1u << q)) {
            const X v = dev::ld_relaxed(x + jj[q]);
            if (!Sentinel<X>::is(v)) {
              xv[q] = v;
              pend &= ~(1u << q);
            }
          }
        if (!pend) {
          X sum = X(0);
#pragma unroll
          for (int q = 0; q < KD; q++)
            if (kb + q < ke)
              sum = add_rn(sum, mul_rn(a[q], xv[q]));
          X xi = sub_rn(__ldg(b + i), sum);
          if (!UNIT)
            xi = div_rn(xi, X(__ldg(diag + p)));
          dev::st_relaxed(x + i, Sentinel<X>::scrub(xi));
          done = true;
        }
      }
      if (__all_sync(0xffffffffu, done))
        break;
      bool abort = false;
      if ((pass & 15u) == 0u && lane == 0)
        abort = dev::ld_relaxed(err) != 0 || global_ns() - t0 > kWaitNs;
      if (__shfl_sync(0xffffffffu, abort, 0)) {
        if (lane == 0)
          atomicExch(err, 1);
        return;
      }
      if (sleep_ns > 0)
        __nanosleep(sleep_ns);
    }
  }
}

// ---------------------------------------------------------------- parts
// Partitioned schedule.  The rows are split into compact parts (value cuts
// on coordinates monotone along the dependencies, la_partition.cpp, so the
// parts' dependency graph is acyclic), one CTA per part, all CTAs
// co-resident (cooperative launch).  A CTA walks the levels present in its
// part in increasing order, one __syncthreads per level, and keeps the x
// values of its own rows in shared memory: a dependency inside the part costs
// a shared-memory read, and only a dependency on another part goes through
// global memory, where it is awaited as in the level-order schedule (the
// sentinel value is its own flag, waits bounded by the global timer).  A
// dependency path crosses each part boundary at most once, so the critical
// path is the number of levels times a shared-memory step plus a few global
// hand-offs, instead of the number of levels times an L2 round trip.
// No deadlock: every CTA is resident and processes its rows in level order,
// so the unfinished row of lowest level always has its inputs ready.
constexpr int kEmptySlot = 0x7fffffff; // column of an unused slot
constexpr int kNoRing = kTrsvNoRing;   // ring_mask when every row has its own slot

// threads per CTA: four prefetched rows live in registers
template <typename X, int KD> constexpr int part_threads() {
  return KD <= 4 ? 512 : 256;
}

template <typename X, int KD> struct PartRow {
  int r, i; // execution position (-1: none) and original row
  int j[KD];
  X a[KD];
  X dg;
  X xr[KD]; // values of other parts' rows, loaded ahead
};

// Nothing but shared-memory reads, arithmetic and the barrier may sit on a
// level's critical path, so everything global is fetched ahead:
//  * the part's level boundaries and the b values of its rows are staged in
//    shared memory at kernel start (row r's x slot holds b until row r
//    overwrites it with x);
//  * 3-slot rows are two records per execution position, {row, 3 columns}
//    (int4) and {3 values, diagonal}; longer rows keep their first KD
//    entries slot-major (ej[s*n + r], ev[s*n + r]); kEmptySlot marks an
//    unused slot.  A warp's rows are coalesced loads either way -- two
//    vector loads a row (three in FP64) against one per slot -- and every
//    thread fetches its first row of level q+3 while it solves level q (four
//    register sets);
//  * at the end of level q it issues the loads of the other parts' values
//    that its level-(q+2) row reads -- two levels after that row's columns
//    were requested, so the addresses are there -- and only re-reads (waits
//    for) those that were not yet published when it gets to them.
// Entries beyond KD (only when some row is longer than 16) come from the CSR
// copy, and rows beyond the first per thread in levels wider than the CTA
// are loaded when reached.
// Ring mode (ring_mask != kNoRing), for parts whose rows do not all fit in
// shared memory: the x slots form a ring of ring_mask + 1 rows, row r of the
// part in slot (r - P0) & ring_mask.  The analysis encodes a dependency on
// the part's own row as a slot only while that slot cannot yet have been
// reused (see build_parts); older ones are read from x in global memory,
// published several barriers earlier.  b is not staged at kernel start:
// each prefetched row's b is copied into its slot by cp.async when the row
// is armed (two levels ahead), and the solve waits for that copy first.
// W2 (FP32, short rows): levels wider than the CTA are common in large parts;
// two more register sets hold each thread's second row of a level, fetched
// at the start of the level before (L2, pulled in by the bulk prefetch) and
// its other parts' values requested at the start of its own level, so the
// second round of a wide level costs no global round trip of its own.
template <typename V, typename X, bool UNIT, int KD, bool W2 = false>
__global__ void __launch_bounds__(part_threads<X, KD>(), 1)
    trsv_part_kernel(const int n, const int *__restrict__ pstart,
                     const int *__restrict__ psub, const int *__restrict__ sb,
                     const int *__restrict__ ai, const int *__restrict__ aj,
                     const V *__restrict__ av, const int *__restrict__ ej,
                     const V *__restrict__ ev, const V *__restrict__ diag,
                     const int *__restrict__ exec_row, const X *__restrict__ b, X *x,
                     int *err, const int tail, const int rows_cap, const int ring_mask,
                     const int4 *__restrict__ rmeta, const V *__restrict__ rval) {
  constexpr int T = part_threads<X, KD>();
  const bool ring = ring_mask != kNoRing;
  extern __shared__ __align__(16) unsigned char part_smem[];
  X *xs = reinterpret_cast<X *>(part_smem);
  int *ssb = reinterpret_cast<int *>(xs + rows_cap); // level boundaries
  const int p = blockIdx.x, tid = threadIdx.x;
  const int P0 = __ldg(pstart + p), P1 = __ldg(pstart + p + 1);
  const int q0 = __ldg(psub + p), q1 = __ldg(psub + p + 1);
  const unsigned long long t0 = global_ns();
  int aborted = 0; // this thread gave up on a wait (or saw another give up)

  auto load_row = [&](int r, PartRow<X, KD> &R) {
    R.r = r;
    if constexpr (KD == 3) { // two records: {row, 3 columns}, {3 values, diagonal}
      const int4 m = dev::ld_ahead(rmeta + r);
      V v[4];
      dev::ld_ahead4(rval + 4 * (size_t)r, v);
      R.i = m.x, R.j[0] = m.y, R.j[1] = m.z, R.j[2] = m.w;
#pragma unroll
      for (int s = 0; s < 3; s++)
        R.a[s] = X(v[s]);
      R.dg = UNIT ? X(1) : X(v[3]);
    } else {
      R.i = dev::ld_ahead(exec_row + r);
#pragma unroll
      for (int s = 0; s < KD; s++) {
        R.j[s] = dev::ld_ahead(ej + (size_t)s * n + r);
        R.a[s] = X(dev::ld_ahead(ev + (size_t)s * n + r));
      }
      R.dg = UNIT ? X(1) : X(dev::ld_ahead(diag + r));
    }
  };
  auto prefetch = [&](int q, PartRow<X, KD> &R) {
    R.r = -1;
    if (q < q1) {
      const int r = ssb[q - q0] + tid;
      if (r < ssb[q - q0 + 1])
        load_row(r, R);
    }
  };
  auto arm = [&](PartRow<X, KD> &R) {
    if (R.r >= 0) {
#pragma unroll
      for (int s = 0; s < KD; s++)
        if (R.j[s] >= 0 && R.j[s] != kEmptySlot)
          R.xr[s] = dev::ld_relaxed(x + R.j[s]);
      if (ring)
        dev::cp_async_shared(xs + ((R.r - P0) & ring_mask), b + R.i);
    }
    if (ring) // one group per armed level, empty or not
      dev::cp_async_commit();
  };
  // a value of another part: wait (bounded) until it stops being the sentinel
  auto await = [&](int c, X v) {
    for (unsigned pass = 1; Sentinel<X>::is(v) && !aborted; pass++) {
      if ((pass & 63u) == 0u && (dev::ld_relaxed(err) != 0 || global_ns() - t0 > kWaitNs)) {
        atomicExch(err, 1);
        aborted = 1;
      }
      v = dev::ld_relaxed(x + c);
    }
    return v;
  };
  // The slot reads are issued together (no branch between them), values of
  // other parts that were not yet published are waited for afterwards (the
  // rare case), and only then is the row summed in stored order -- an unused
  // slot adds nothing, so the result is the reference's bit for bit.
  // b_in_slot: b was staged at kernel start (whole parts) or copied in when
  // the row was armed (ring mode); otherwise it is read here
  auto solve_row = [&](const PartRow<X, KD> &R, bool armed, bool b_in_slot) {
    const int slot = (R.r - P0) & ring_mask;
    const X bi = b_in_slot ? xs[slot] : __ldg(b + R.i);
    X v[KD];
#pragma unroll
    for (int s = 0; s < KD; s++) {
      const int c = R.j[s];
      v[s] = c < 0 ? xs[-1 - c] : (armed ? R.xr[s] : X(0));
    }
#pragma unroll
    for (int s = 0; s < KD; s++) {
      const int c = R.j[s];
      if (c >= 0 && c != kEmptySlot && (!armed || Sentinel<X>::is(v[s])))
        v[s] = await(c, armed ? v[s] : dev::ld_relaxed(x + c));
    }
    X sum = X(0);
#pragma unroll
    for (int s = 0; s < KD; s++)
      sum = R.j[s] != kEmptySlot ? add_rn(sum, mul_rn(R.a[s], v[s])) : sum;
    if (tail) {
      const int k1 = __ldg(ai + R.r + 1);
      for (int k = __ldg(ai + R.r) + KD; k < k1; k++) {
        const int c = __ldg(aj + k);
        const X v = c < 0 ? xs[-1 - c] : await(c, dev::ld_relaxed(x + c));
        sum = add_rn(sum, mul_rn(X(__ldg(av + k)), v));
      }
    }
    X xi = sub_rn(bi, sum);
    if (!UNIT)
      xi = div_rn(xi, R.dg);
    xs[slot] = xi;
    dev::st_relaxed(x + R.i, Sentinel<X>::scrub(xi));
  };
  // W2: a thread's second row of level q (r = level start + T + tid)
  auto prefetch2 = [&](int q, PartRow<X, KD> &S) {
    S.r = -1;
    if (q < q1) {
      const int r = ssb[q - q0] + T + tid;
      if (r < ssb[q - q0 + 1])
        load_row(r, S);
    }
  };
  auto arm2 = [&](PartRow<X, KD> &S) {
    if (S.r >= 0) {
#pragma unroll
      for (int s = 0; s < KD; s++)
        if (S.j[s] >= 0 && S.j[s] != kEmptySlot)
          S.xr[s] = dev::ld_relaxed(x + S.j[s]);
    }
  };
  auto run_level = [&](int q, const PartRow<X, KD> &R, PartRow<X, KD> &Sc,
                       PartRow<X, KD> &Sn) {
    if (ring) // this row's b copy: all but the newest group (level q+1's) are done
      dev::cp_async_wait_all_but_one();
    if (W2) {
      prefetch2(q + 1, Sn);
      arm2(Sc);
    }
    if (R.r < 0)
      return;
    solve_row(R, true, true);
    const int e = ssb[q - q0 + 1];
    int r = R.r + T;
    if (W2 && Sc.r >= 0) {
      solve_row(Sc, true, !ring);
      r += T;
    }
    for (; r < e; r += T) { // levels wider than the CTA
      PartRow<X, KD> S;
      load_row(r, S);
      solve_row(S, false, !ring);
    }
  };

  for (int q = q0 + tid; q <= q1; q += T)
    ssb[q - q0] = __ldg(sb + q);
  __syncthreads();
  // Slices of the row arrays are pulled into L2 several levels ahead, four
  // levels per fire-and-forget bulk prefetch, one array per warp, so the
  // register fetch three levels ahead reads L2 rather than HBM.
  auto l2_ahead = [&](int q, int qe) { // levels [q, qe) of the part
    const int a = tid >> 5;
    qe = min(qe, q1);
    if ((tid & 31) != 0 || a >= 2 * KD + 2 || q >= qe)
      return;
    const int s = ssb[q - q0], e = ssb[qe - q0];
    const char *base_ptr;
    size_t es;
    if constexpr (KD == 3) { // the two record arrays
      if (a >= 2)
        return;
      base_ptr = a == 0 ? reinterpret_cast<const char *>(rmeta)
                        : reinterpret_cast<const char *>(rval);
      es = a == 0 ? sizeof(int4) : 4 * sizeof(V);
    } else if (a == 0) {
      base_ptr = reinterpret_cast<const char *>(exec_row);
      es = 4;
    } else if (a == 1) {
      base_ptr = reinterpret_cast<const char *>(diag);
      es = sizeof(V);
      if (UNIT)
        return;
    } else if (a < 2 + KD) {
      base_ptr = reinterpret_cast<const char *>(ej + (size_t)(a - 2) * n);
      es = 4;
    } else {
      base_ptr = reinterpret_cast<const char *>(ev + (size_t)(a - 2 - KD) * n);
      es = sizeof(V);
    }
    // a bulk prefetch needs a 16-byte aligned address and size: round the
    // absolute range outwards (allocations are 256-byte aligned and padded by
    // 64 bytes, so this stays inside them)
    const size_t lo = reinterpret_cast<size_t>(base_ptr + (size_t)s * es) & ~(size_t)15;
    const size_t hi = (reinterpret_cast<size_t>(base_ptr + (size_t)e * es) + 15) & ~(size_t)15;
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(lo),
                 "r"((unsigned)(hi - lo))
                 : "memory");
  };
  PartRow<X, KD> R0, R1, R2, R3;
  PartRow<X, KD> S0, S1; // W2 only
  S0.r = S1.r = -1;
  l2_ahead(q0 + 3, q0 + 8);
  prefetch(q0, R0);
  prefetch(q0 + 1, R1);
  prefetch(q0 + 2, R2);
  // b of the part's rows into their x slots, 16 rows per thread per batch
  // (all row indices, then all b values, in flight together)
  constexpr int kStage = 16;
  for (int r0 = P0 + tid; !ring && r0 < P1; r0 += kStage * T) {
    int ii[kStage];
    X bv[kStage];
#pragma unroll
    for (int u = 0; u < kStage; u++)
      ii[u] = r0 + u * T < P1 ? __ldg(exec_row + r0 + u * T) : -1;
#pragma unroll
    for (int u = 0; u < kStage; u++)
      bv[u] = ii[u] >= 0 ? __ldg(b + ii[u]) : X(0);
#pragma unroll
    for (int u = 0; u < kStage; u++)
      if (ii[u] >= 0)
        xs[r0 + u * T - P0] = bv[u];
  }
  __syncthreads();
  arm(R0);
  arm(R1);
  if (W2)
    prefetch2(q0, S0);
  // four register sets rotate: level q runs, then q+2 is armed and q+3 is
  // fetched (after the solve, so its loads do not delay the solve's reads);
  // one barrier per level, and every thread leaves together if any gave up
  for (int q = q0; q < q1; q += 4) {
    run_level(q, R0, S0, S1);
    arm(R2);
    l2_ahead(q + 8, q + 12); // four levels per bulk prefetch
    prefetch(q + 3, R3);
    if (__syncthreads_or(aborted) || q + 1 >= q1)
      break;
    run_level(q + 1, R1, S1, S0);
    arm(R3);
    prefetch(q + 4, R0);
    if (__syncthreads_or(aborted) || q + 2 >= q1)
      break;
    run_level(q + 2, R2, S0, S1);
    arm(R0);
    prefetch(q + 5, R1);
    if (__syncthreads_or(aborted) || q + 3 >= q1)
      break;
    run_level(q + 3, R3, S1, S0);
    arm(R1);
    prefetch(q + 6, R2);
    if (__syncthreads_or(aborted))
      break;
  }
  if (ring) // no copy may still be landing when the CTA leaves (an abort)
    dev::cp_async_wait_all();
}

template <typename V, typename X, bool UNIT>
void launch_kernel(la_trsv_plan_t P, const X *b, X *x, cudaStream_t st) {
  const int *cs = P->chunk_start.as<int>(), *ai = P->ai.as<int>(),
            *aj = P->aj.as<int>(), *er = P->exec_row.as<int>();
  const V *av = P->av.as<V>(), *dg = P->diag.as<V>();
  int *err = P->err.as<int>(), *tk = P->ticket.as<int>();
  const dim3 g(P->grid), t(kThreads);
  switch (P->kd) {
  case 4:
    trsv_level_kernel<V, X, UNIT, 4><<<g, t, 0, st>>>(P->nchunks, cs, ai, aj, av, dg, er, b,
                                                      x, P->base, err, tk, P->sleep_ns);
    break;
  case 8:
    trsv_level_kernel<V, X, UNIT, 8><<<g, t, 0, st>>>(P->nchunks, cs, ai, aj, av, dg, er, b,
                                                      x, P->base, err, tk, P->sleep_ns);
    break;
  case 16:
    trsv_level_kernel<V, X, UNIT, 16><<<g, t, 0, st>>>(P->nchunks, cs, ai, aj, av, dg, er,
                                                       b, x, P->base, err, tk, P->sleep_ns);
    break;
  default:
    trsv_level_kernel_grouped<V, X, UNIT><<<g, t, 0, st>>>(P->nchunks, cs, ai, aj, av, dg,
                                                           er, b, x, P->base, err, tk);
  }
}

template <typename V, typename X, bool UNIT, int KD, bool W2 = false>
const void *part_fn() {
  return (const void *)trsv_part_kernel<V, X, UNIT, KD, W2>;
}

template <typename V, typename X, bool UNIT, int KD, bool W2 = false>
cudaError_t launch_parts_kd(la_trsv_plan_t P, const X *b, X *x, cudaStream_t st) {
  const int n = P->n, tail = P->kd == 0;
  const int *ps = P->pstart.as<int>(), *pq = P->psub.as<int>(), *sb = P->sb.as<int>(),
            *ai = P->ai.as<int>(), *aj = P->aj.as<int>(), *ej = P->ej.as<int>(),
            *er = P->exec_row.as<int>();
  const V *av = P->av.as<V>(), *ev = P->ev.as<V>(), *dg = P->diag.as<V>();
  int *err = P->err.as<int>();
  const int cap = P->part_rows, mask = P->ring_mask;
  const int4 *rm = P->rmeta.as<int4>();
  const V *rv = P->rval.as<V>();
  void *args[] = {(void *)&n,  (void *)&ps, (void *)&pq, (void *)&sb,  (void *)&ai,
                  (void *)&aj, (void *)&av, (void *)&ej, (void *)&ev,  (void *)&dg,
                  (void *)&er, (void *)&b,  (void *)&x,  (void *)&err, (void *)&tail,
                  (void *)&cap, (void *)&mask, (void *)&rm, (void *)&rv};
  return cudaLaunchCooperativeKernel(part_fn<V, X, UNIT, KD, W2>(), dim3(P->nparts),
                                     dim3(part_threads<X, KD>()), args, P->part_smem, st);
}

template <typename V, typename X, bool UNIT>
cudaError_t launch_parts(la_trsv_plan_t P, const X *b, X *x, cudaStream_t st) {
  if constexpr (sizeof(X) == 4)
    if (P->w2 && P->kd == 3)
      return launch_parts_kd<V, X, UNIT, 3, true>(P, b, x, st);
  switch (P->kd) {
  case 3:
    return launch_parts_kd<V, X, UNIT, 3>(P, b, x, st);
  case 4:
    return launch_parts_kd<V, X, UNIT, 4>(P, b, x, st);
  case 8:
    return launch_parts_kd<V, X, UNIT, 8>(P, b, x, st);
  default: // 16 slots; longer rows finish from the CSR tail
    return launch_parts_kd<V, X, UNIT, 16>(P, b, x, st);
  }
}

template <typename V, typename X>
la_status launch_typed(la_trsv_plan_t P, const X *b, X *x, cudaStream_t st) {
  if (P->n == 0)
    return LA_OK;
  LA_CUDA_TRY(cudaMemsetAsync(x, 0xff, sizeof(X) * (size_t)P->n, st));
  if (P->sched == 1) {
    const cudaError_t e = P->unit ? launch_parts<V, X, true>(P, b, x, st)
                                  : launch_parts<V, X, false>(P, b, x, st);
    LA_CUDA_TRY(e);
    return LA_OK;
  }
  LA_CUDA_TRY(cudaMemsetAsync(P->ticket.p, 0, sizeof(int), st));
  if (P->unit)
    launch_kernel<V, X, true>(P, b, x, st);
  else
    launch_kernel<V, X, false>(P, b, x, st);
  LA_CUDA_TRY(cudaGetLastError());
  return LA_OK;
}

// Persistent grid: a few CTAs per SM (LA_TRSV_CTAS_PER_SM overrides the
// default of 2), capped by occupancy and by the number of chunks.  More
// warps than the widest levels can use only add polling traffic.
template <typename V, typename X> int grid_for(int nchunks, int kd) {
  const void *fns[2];
  switch (kd) {
  case 4:
    fns[0] = (const void *)trsv_level_kernel<V, X, false, 4>;
    fns[1] = (const void *)trsv_level_kernel<V, X, true, 4>;
    break;
  case 8:
    fns[0] = (const void *)trsv_level_kernel<V, X, false, 8>;
    fns[1] = (const void *)trsv_level_kernel<V, X, true, 8>;
    break;
  case 16:
    fns[0] = (const void *)trsv_level_kernel<V, X, false, 16>;
    fns[1] = (const void *)trsv_level_kernel<V, X, true, 16>;
    break;
  default:
    fns[0] = (const void *)trsv_level_kernel_grouped<V, X, false>;
    fns[1] = (const void *)trsv_level_kernel_grouped<V, X, true>;
  }
  int fit = 1 << 30;
  for (const void *f : fns) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, f, kThreads, 0);
    fit = std::min(fit, std::max(1, per_sm));
  }
  int want = 2;
  if (const char *e = std::getenv("LA_TRSV_CTAS_PER_SM"))
    want = std::max(1, std::atoi(e));
  const int g = std::min(want, fit) * sm_count();
  const int need = (nchunks + kThreads / 32 - 1) / (kThreads / 32);
  return std::max(1, std::min(g, need));
}

} // namespace

la_status trsv_launch(la_trsv_plan_t P, const void *b, void *x,
                      cudaStream_t st) {
  if (P->dtype == LA_F64)
    return launch_typed<double, double>(P, (const double *)b, (double *)x, st);
  return launch_typed<float, float>(P, (const float *)b, (float *)x, st);
}

// The plans of one preconditioner (L and U = L^T, FP64 and FP32) share one
// undirected graph, and a partition computed for one of them is valid for
// all: the solve is correct for any partition, landmark coordinates are
// monotone whatever the edges' direction, and L's level order is monotone
// (reversed) for U.  So the last few partitions are kept, keyed by the row
// count, the part count and an order-independent hash of the graph's edges.
std::mutex g_part_mu;
struct PartEntry {
  int n, nparts;
  unsigned long long hash;
  std::vector<int> part;
};
std::vector<PartEntry> g_part_cache; // most recent last, at most 4

void cached_partition(int n, const int *ai, const int *aj, int base,
                      const std::vector<int> &lvl, int nparts, std::vector<int> &part) {
  // the key: a sum over the stored entries, each hashed as its undirected
  // edge (smaller row first) -- the same for a triangle and its transpose,
  // independent of the order, and computed in parallel (integer sums)
  unsigned long long h = 0x9e3779b97f4a7c15ull * (unsigned long long)(n + 1);
#pragma omp parallel for schedule(static) reduction(+ : h)
  for (int i = 0; i < n; i++)
    for (int k = ai[i] - base; k < ai[i + 1] - base; k++) {
      const int j = aj[k] - base;
      const unsigned long long a = (unsigned long long)std::min(i, j),
                               b = (unsigned long long)std::max(i, j);
      unsigned long long z = a * 0x100000001b3ull ^ b;
      z = (z ^ (z >> 31)) * 0xbf58476d1ce4e5b9ull;
      h += z ^ (z >> 29);
    }
  {
    std::lock_guard<std::mutex> lock(g_part_mu);
    for (const PartEntry &e : g_part_cache)
      if (e.n == n && e.nparts == nparts && e.hash == h) {
        part = e.part;
        return;
      }
  }
  // the landmark stage on the GPU; should a device step fail (memory), the
  // host's stage gives the same parts
  part.assign(n, 0);
  la_status st = LA_OK;
  if (monotone_partition_device(n, base, ai, aj, lvl.data(), nparts, part.data(), &st) < 0) {
    cudaGetLastError();
    std::vector<int> xadj, adj;
    undirected_pattern(n, base, ai, aj, xadj, adj);
    monotone_partition(n, xadj.data(), adj.data(), ai, aj, base, lvl.data(), nparts,
                       part.data());
  }
  std::lock_guard<std::mutex> lock(g_part_mu);
  if (g_part_cache.size() == 4)
    g_part_cache.erase(g_part_cache.begin());
  g_part_cache.push_back({n, nparts, h, part});
}

// Partitioned layout (schedule 1).  Leaves the plan untouched and reports
// *ok = false when the device cannot keep one CTA per part resident, or when
// a part's rows fit in shared memory neither whole nor as a ring (ring mode
// needs any three consecutive levels of a part to fit).
template <typename X>
la_status build_parts(la_trsv_plan_t P, const int *ai, const int *aj, const double *av,
                      const double *diag, bool force, bool *ok) {
  *ok = false;
  const int n = P->n, base = P->base, nnz = P->nnz;
  int dev = 0, optin = 0;
  LA_CUDA_TRY(cudaGetDevice(&dev));
  LA_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  // a power of two: the k-d cuts then halve every node evenly (measured, 128
  // against 148 parts: 128^3 factor 0.303 / 0.460 ms against 0.310 / 0.470
  // FP32 / FP64, 192^3 FP32 0.796 against 0.814 ms; 136 or 144 in between)
  int nparts = std::min(sm_count(), std::max(1, (n + 2047) / 2048));
  while (nparts & (nparts - 1))
    nparts &= nparts - 1;
  if (const char *e = std::getenv("LA_TRSV_PARTS")) // tuning override
    nparts = std::max(1, std::min(sm_count(), std::atoi(e)));
  // rows' levels, then the partition (of the triangle's graph made undirected)
  std::vector<int> lvl(n);
#pragma omp parallel for schedule(dynamic, 16)
  for (int l = 0; l < P->levels; l++)
    for (int p = P->h_prefix[l]; p < P->h_prefix[l + 1]; p++)
      lvl[P->h_iperm[p] - base] = l;
  std::vector<int> part;
  cached_partition(n, ai, aj, base, lvl, nparts, part);
  // The layout's host loops run over fixed chunks of the execution order on
  // the host's threads; every array is the one a serial pass writes.
  constexpr int kChunkRows = 1 << 16;
  const int nchunk = (n + kChunkRows - 1) / kChunkRows;
  // per chunk and part: rows of the part in the chunk (execution order)
  std::vector<int> ccount((size_t)nchunk * nparts, 0);
  int longest = 0; // register slots from the longest row (16 plus the CSR tail beyond)
#pragma omp parallel for schedule(static) reduction(max : longest)
  for (int c = 0; c < nchunk; c++) {
    int *cc = ccount.data() + (size_t)c * nparts;
    for (int q = c * kChunkRows; q < std::min(n, (c + 1) * kChunkRows); q++) {
      const int i = P->h_iperm[q] - base;
      cc[part[i]]++;
      longest = std::max(longest, ai[i + 1] - ai[i]);
    }
  }
  std::vector<int> pstart(nparts + 1, 0);
  for (int c = 0; c < nchunk; c++)
    for (int p = 0; p < nparts; p++)
      pstart[p + 1] += ccount[(size_t)c * nparts + p];
  int rows_max = 0;
  for (int p = 0; p < nparts; p++)
    rows_max = std::max(rows_max, pstart[p + 1]);
  std::partial_sum(pstart.begin(), pstart.end(), pstart.begin());
  // (3 slots for the 7-point stencils' IC(0) factors: a fourth would hold four
  // registers per prefetched row for nothing, and FP64 needs them)
  const int kd = longest <= 3 ? 3 : longest <= 4 ? 4 : longest <= 8 ? 8 : longest <= 16 ? 16 : 0;
  const int ks = kd ? kd : 16;
  // execution order: part-major, level order inside a part (a stable
  // counting sort of the level order by part: chunk c's rows of part p start
  // after those of the earlier chunks); sb = the start position of every
  // (part, level), psub = each part's first entry
  // (every entry written below: left uninitialised, no first-touch pass)
  std::unique_ptr<int[]> erow(new int[std::max(n, 1)]), pos(new int[std::max(n, 1)]);
  {
    for (int p = 0; p < nparts; p++) { // ccount becomes each chunk's first slot
      int at = pstart[p];
      for (int c = 0; c < nchunk; c++) {
        const int k = ccount[(size_t)c * nparts + p];
        ccount[(size_t)c * nparts + p] = at;
        at += k;
      }
    }
#pragma omp parallel for schedule(static)
    for (int c = 0; c < nchunk; c++) {
      int *fill = ccount.data() + (size_t)c * nparts;
      for (int q = c * kChunkRows; q < std::min(n, (c + 1) * kChunkRows); q++) {
        const int i = P->h_iperm[q] - base, r = fill[part[i]]++;
        erow[r] = i;
        pos[i] = r;
      }
    }
  }
  std::vector<int> nsub(nparts, 0), psub(nparts + 1);
  std::unique_ptr<int[]> lvl_at(new int[std::max(n, 1)]);
#pragma omp parallel for schedule(dynamic, 1)
  for (int p = 0; p < nparts; p++)
    for (int r = pstart[p]; r < pstart[p + 1]; r++)
      nsub[p] += r == pstart[p] || lvl[erow[r]] != lvl[erow[r - 1]];
  int subs_max = 0;
  psub[0] = 0;
  for (int p = 0; p < nparts; p++) {
    psub[p + 1] = psub[p] + nsub[p];
    subs_max = std::max(subs_max, nsub[p]);
  }
  std::vector<int> sb(psub[nparts] + 1);
#pragma omp parallel for schedule(dynamic, 1)
  for (int p = 0; p < nparts; p++) {
    int g = psub[p] - 1;
    for (int r = pstart[p]; r < pstart[p + 1]; r++) {
      if (r == pstart[p] || lvl[erow[r]] != lvl[erow[r - 1]])
        sb[++g] = r;
      lvl_at[r] = g;
    }
  }
  sb[psub[nparts]] = n;
  // end of the level two after the one at sb index g (part p)
  auto end2 = [&](int p, int g) { return sb[std::min(g + 3, psub[p + 1])]; };
  // shared memory: every row of the largest part, else a ring (power of two)
  const size_t sb_bytes = sizeof(int) * ((size_t)subs_max + 1);
  int ring = 0; // ring rows, 0 = whole parts
  if (sizeof(X) * (size_t)rows_max + sb_bytes + 1024 > (size_t)optin) {
    if (sb_bytes + 1024 + sizeof(X) * 1024 > (size_t)optin)
      return LA_OK;
    ring = 1024;
    while (sizeof(X) * (size_t)ring * 2 + sb_bytes + 1024 <= (size_t)optin)
      ring *= 2;
  }
  if (const char *e = std::getenv("LA_TRSV_RING")) { // testing / tuning override
    const int r = std::atoi(e);
    if (r >= 32 && (r & (r - 1)) == 0 && sizeof(X) * (size_t)r + sb_bytes + 1024 <= (size_t)optin)
      ring = r;
  }
  if (ring)
    for (int p = 0; p < nparts; p++)
      for (int g = psub[p]; g < psub[p + 1]; g++)
        if (end2(p, g) - sb[g] > ring)
          return LA_OK; // three consecutive levels must fit in the ring
  const size_t smem = sizeof(X) * (size_t)(ring ? ring : rows_max) + sb_bytes;
  const void *fns[2];
  int threads = 0;
  // second-row register sets when some level of a part is wider than the
  // CTA (FP32 3-slot rows: the only variant whose registers allow them)
  int widest = 0;
  for (int g = 0; g < psub[nparts]; g++)
    widest = std::max(widest, sb[g + 1] - sb[g]);
  bool w2 = false;
  if constexpr (sizeof(X) == 4) {
    w2 = ks == 3 && widest > part_threads<X, 3>();
    if (const char *e = std::getenv("LA_TRSV_W2")) // testing / tuning override
      w2 = w2 && std::atoi(e) != 0;
    if (w2) {
      fns[0] = part_fn<X, X, false, 3, true>(), fns[1] = part_fn<X, X, true, 3, true>();
      threads = part_threads<X, 3>();
    }
  }
  if (w2) {
    // fns and threads set above
  } else if (ks == 3) {
    fns[0] = part_fn<X, X, false, 3>(), fns[1] = part_fn<X, X, true, 3>();
    threads = part_threads<X, 3>();
  } else if (ks == 4) {
    fns[0] = part_fn<X, X, false, 4>(), fns[1] = part_fn<X, X, true, 4>();
    threads = part_threads<X, 4>();
  } else if (ks == 8) {
    fns[0] = part_fn<X, X, false, 8>(), fns[1] = part_fn<X, X, true, 8>();
    threads = part_threads<X, 8>();
  } else {
    fns[0] = part_fn<X, X, false, 16>(), fns[1] = part_fn<X, X, true, 16>();
    threads = part_threads<X, 16>();
  }
  for (const void *f : fns) {
    // the limit is per kernel, shared by every plan: allow the device's
    // maximum once, so that a smaller plan never lowers a larger plan's limit
    if (cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, optin) !=
        cudaSuccess) {
      cudaGetLastError();
      return LA_OK;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, f, threads, smem) !=
            cudaSuccess ||
        (long long)per_sm * sm_count() < nparts) {
      cudaGetLastError();
      return LA_OK;
    }
  }
  // Modelled critical path (microseconds; B200 measurements): a part takes
  // ~0.35 us per level it holds plus ~1 us for every further round of rows
  // in a level wider than its CTA (~0.3 us for the second round when it is
  // held in registers, W2), both 1.2x for FP64 3-slot rows and 1.5x for
  // longer FP64 rows (a part's level step measured 0.96 / 1.24 us FP64 --
  // with / without the 3-slot row records -- against 0.79 / 0.80 us FP32 on
  // the 128^3 IC(0) factor, while the level order costs about the same in
  // both; with the factor 1.2 the 192^3 FP64 factor's ring-mode parts,
  // 1.107 ms, are taken over its level order, 1.201 ms), and a value
  // crossing parts arrives ~1.5 us after it is written; the level-order
  // schedule takes ~2 us per level.  The partition is used when it models
  // at most 0.8 of that.
  if (!force) {
    const double f = sizeof(X) == 8 ? (kd == 3 ? 1.2 : 1.5) : 1.0;
    std::vector<double> ready(n), last(nparts, 0.0), fin(nparts, 0.0), tin;
    std::vector<int> width(nparts, 0), touched;
    // a row's input time: the latest of its dependencies' (levels of 4096
    // rows or more on the host's threads; a max, so the same in any order)
    auto input_time = [&](int q) {
      const int i = P->h_iperm[q] - base, pi = part[i];
      double t = 0;
      for (int k = ai[i] - base; k < ai[i + 1] - base; k++) {
        const int j = aj[k] - base;
        t = std::max(t, ready[j] + (part[j] != pi ? 1.5 : 0.0));
      }
      return t;
    };
    for (int l = 0; l < P->levels; l++) {
      touched.clear();
      const int q0l = P->h_prefix[l], q1l = P->h_prefix[l + 1];
      const bool wide = q1l - q0l >= 4096;
      if (wide) {
        tin.resize(q1l - q0l);
#pragma omp parallel for schedule(static)
        for (int q = q0l; q < q1l; q++)
          tin[q - q0l] = input_time(q);
      }
      for (int q = q0l; q < q1l; q++) {
        const int i = P->h_iperm[q] - base, pi = part[i];
        const double t = wide ? tin[q - q0l] : input_time(q);
        if (width[pi]++ == 0) {
          touched.push_back(pi);
          fin[pi] = last[pi];
        }
        fin[pi] = std::max(fin[pi], t);
      }
      for (int p : touched) {
        const int extra = (width[p] + threads - 1) / threads - 1;
        const double rounds = w2 && extra > 0 ? 0.3 + 1.0 * (extra - 1) : 1.0 * extra;
        fin[p] += f * (0.35 + rounds);
      }
      for (int q = P->h_prefix[l]; q < P->h_prefix[l + 1]; q++) {
        const int i = P->h_iperm[q] - base;
        ready[i] = fin[part[i]];
      }
      for (int p : touched) {
        last[p] = fin[p];
        width[p] = 0;
      }
    }
    double est = 0;
    for (int p = 0; p < nparts; p++)
      est = std::max(est, last[p]);
    if (est > 0.8 * 2.0 * P->levels)
      return LA_OK;
  }
  // encoded columns (-1 - x slot for the part's own rows), first ks entries
  // slot-major, all entries in CSR for rows beyond ks.  In ring mode a row r
  // of level g reads its part's row d from the ring only if d >= end of level
  // g + 2 minus the ring size: d's slot is refilled by row d + ring, whose b
  // is copied in while level (d + ring's level) - 2 is still being solved, so
  // d + ring must lie beyond level g + 2.  Older rows are read from x.
  // Values go straight into the solve's type X (the same rounding as a
  // conversion afterwards).  Scratch is left uninitialised: each row writes
  // all of its own cells, on the host's threads.
  const size_t cells = (size_t)ks * n;
  std::unique_ptr<int[]> ej(new int[cells]);
  std::unique_ptr<X[]> ev(new X[cells]), ediag(new X[std::max(n, 1)]);
  std::vector<int> eai;
  std::unique_ptr<int[]> eaj;
  std::unique_ptr<X[]> eav;
  if (!kd) {
    eai.assign(n + 1, 0);
    for (int r = 0; r < n; r++)
      eai[r + 1] = eai[r] + (ai[erow[r] + 1] - ai[erow[r]]);
    eaj.reset(new int[std::max(nnz, 1)]);
    eav.reset(new X[std::max(nnz, 1)]);
  }
#pragma omp parallel for schedule(dynamic, 4096)
  for (int r = 0; r < n; r++) {
    const int i = erow[r], pi = part[i];
    ediag[r] = diag ? (X)diag[i] : (X)1;
    for (int s = 0; s < ks; s++) {
      ej[(size_t)s * n + r] = kEmptySlot;
      ev[(size_t)s * n + r] = (X)0;
    }
    int w = kd ? 0 : eai[r];
    for (int k = ai[i] - base, s = 0; k < ai[i + 1] - base; k++, s++, w++) {
      const int j = aj[k] - base;
      int c = j;
      if (part[j] == pi) {
        const int d = pos[j];
        if (!ring)
          c = -1 - (d - pstart[pi]);
        else if (d >= end2(pi, lvl_at[r]) - ring)
          c = -1 - ((d - pstart[pi]) & (ring - 1));
      }
      if (s < ks) {
        ej[(size_t)s * n + r] = c;
        ev[(size_t)s * n + r] = (X)av[k];
      }
      if (!kd) {
        eaj[w] = c;
        eav[w] = (X)av[k];
      }
    }
  }
  if (!kd) {
    LA_TRY(P->ai.upload(eai.data(), sizeof(int) * eai.size()));
    LA_TRY(P->aj.upload(eaj.get(), sizeof(int) * std::max(nnz, 1)));
    LA_TRY(P->av.upload(eav.get(), sizeof(X) * std::max(nnz, 1)));
  }
  // Testing override (the partitioned kernel's bounded wait): the first row
  // with a stored entry reads its own value through global memory instead,
  // a value it publishes only after that read -- so the wait runs out after
  // its 1 s bound and the solve reports LA_ERR_TIMEOUT.
  if (const char *e = std::getenv("LA_TRSV_STALL_TEST"))
    if (std::atoi(e) != 0)
      for (int r = 0; r < n; r++)
        if (ej[r] != kEmptySlot) {
          ej[r] = erow[r];
          break;
        }
  if (kd == 3) {
    // 3-slot rows: one 16-byte record {row, columns} and one {values,
    // diagonal} per position, read by two (FP64: three) vector loads instead
    // of eight scalar ones -- fewer loads in flight per thread and level
    const size_t m = 4 * (size_t)std::max(n, 1);
    std::unique_ptr<int[]> meta(new int[m]);
    std::unique_ptr<X[]> vals(new X[m]);
#pragma omp parallel for schedule(static)
    for (int r = 0; r < n; r++) {
      meta[4 * (size_t)r] = erow[r];
      for (int t = 0; t < 3; t++) {
        meta[4 * (size_t)r + 1 + t] = ej[(size_t)t * n + r];
        vals[4 * (size_t)r + t] = ev[(size_t)t * n + r];
      }
      vals[4 * (size_t)r + 3] = ediag[r];
    }
    LA_TRY(P->rmeta.upload(meta.get(), sizeof(int) * m));
    LA_TRY(P->rval.upload(vals.get(), sizeof(X) * m));
    P->ej.release();
    P->ev.release();
  } else {
    LA_TRY(P->ej.upload(ej.get(), sizeof(int) * cells));
    LA_TRY(P->ev.upload(ev.get(), sizeof(X) * cells));
    P->rmeta.release();
    P->rval.release();
  }
  LA_TRY(P->exec_row.upload(erow.get(), sizeof(int) * n));
  LA_TRY(P->pstart.upload(pstart.data(), sizeof(int) * pstart.size()));
  LA_TRY(P->psub.upload(psub.data(), sizeof(int) * psub.size()));
  LA_TRY(P->sb.upload(sb.data(), sizeof(int) * sb.size()));
  LA_TRY(P->diag.upload(ediag.get(), sizeof(X) * n));
  P->kd = kd;
  P->nparts = nparts;
  P->part_rows = ring ? ring : rows_max;
  P->ring_mask = ring ? ring - 1 : kNoRing;
  P->w2 = w2;
  P->part_smem = smem;
  P->sched = 1;
  *ok = true;
  return LA_OK;
}

// Analysis: TopologicalSort2 levels, rows in execution order, 32-row chunks
// that never cross a level (triangle_solve.tpp:17-113 equivalent).
// A caller-supplied level structure (iperm/prefix as TopologicalSort2
// returns them) replaces the computed one when `iperm` is non-null.
la_status trsv_build(la_trsv_plan_t P, const int *ai, const int *aj,
                     const double *av, const double *diag, const int *iperm,
                     const int *prefix, int nlevels) {
  const int n = P->n, base = P->base;
  if (iperm) {
    P->levels = nlevels;
    P->h_iperm.assign(iperm, iperm + n);
    P->h_prefix.assign(prefix, prefix + nlevels + 1);
  } else {
    P->h_iperm.resize(n);
    P->h_prefix.resize(n + 1);
    // large triangles: the same level sets computed on the GPU
    if (n >= kDeviceLevelsRows) {
      LA_TRY(topological_sort2_device(P->uplo, n, base, ai, aj, P->h_iperm.data(),
                                      P->h_prefix.data(), &P->levels));
    } else {
      P->levels = n == 0 ? 0
                         : topological_sort2(P->uplo, n, base, ai, aj, P->h_iperm.data(),
                                             P->h_prefix.data());
    }
    P->h_prefix.resize(P->levels + 1);
  }
  if (n == 0)
    return LA_OK;
  LA_TRY(P->err.alloc(sizeof(int)));
  LA_CUDA_TRY(cudaMemset(P->err.p, 0, sizeof(int)));
  LA_TRY(P->ticket.alloc(sizeof(int)));
  // The partitioned schedule needs true level sets: every row reads only
  // rows of earlier levels (TopologicalSort2's are by construction; a
  // caller-built structure is checked here and otherwise keeps the
  // level-order schedule, whose bounded waits report a broken order).
  bool exact = true;
  if (iperm) {
    std::vector<int> lvl(n);
    for (int l = 0; l < P->levels; l++)
      for (int p = P->h_prefix[l]; p < P->h_prefix[l + 1]; p++)
        lvl[P->h_iperm[p] - base] = l;
    for (int i = 0; i < n && exact; i++)
      for (int k = ai[i] - base; k < ai[i + 1] - base; k++)
        if (lvl[aj[k] - base] >= lvl[i]) {
          exact = false;
          break;
        }
  }
  // LA_TRSV_SCHEDULE=flags keeps the level-order schedule, =parts takes the
  // partitioned one whenever it fits (both compute bit-identical results)
  const char *sched_env = std::getenv("LA_TRSV_SCHEDULE");
  const bool want_parts = exact && !(sched_env && std::strcmp(sched_env, "flags") == 0);
  const bool force_parts = sched_env && std::strcmp(sched_env, "parts") == 0;
  if (want_parts) {
    bool ok = false;
    LA_TRY(P->dtype == LA_F64 ? build_parts<double>(P, ai, aj, av, diag, force_parts, &ok)
                              : build_parts<float>(P, ai, aj, av, diag, force_parts, &ok));
    if (ok)
      return LA_OK;
  }
  if (const char *e = std::getenv("LA_TRSV_SLEEP_NS")) // tuning override
    P->sleep_ns = std::max(0, std::atoi(e));
  std::vector<int> cstart;
  // filled below on the host's threads, every entry written: no initialisation
  // (zeroed vectors would cost a serial first-touch pass over their pages)
  std::unique_ptr<int[]> eai(new int[n + 1]), erow(new int[std::max(n, 1)]);
  std::unique_ptr<int[]> eaj(new int[std::max(P->nnz, 1)]);
  std::unique_ptr<double[]> eav(new double[std::max(P->nnz, 1)]);
  std::unique_ptr<double[]> ediag(new double[std::max(n, 1)]);
  eaj[0] = 0; // the one placeholder entry of an empty triangle
  eav[0] = 0;
  // row pointers in execution order: row lengths, then a chunked prefix sum
  // (chunk totals added in order), on the host's threads
  eai[0] = base;
  int longest = 0;
#pragma omp parallel for schedule(static) reduction(max : longest)
  for (int p = 0; p < n; p++) {
    const int i = P->h_iperm[p] - base;
    erow[p] = i;
    eai[p + 1] = ai[i + 1] - ai[i];
    longest = std::max(longest, eai[p + 1]);
  }
  {
    constexpr int kScanChunk = 1 << 16;
    const int nc = (n + kScanChunk - 1) / kScanChunk;
    std::vector<int> total(nc + 1, 0);
#pragma omp parallel for schedule(static)
    for (int c = 0; c < nc; c++) {
      int acc = 0;
      for (int p = c * kScanChunk; p < std::min(n, (c + 1) * kScanChunk); p++)
        acc += eai[p + 1];
      total[c + 1] = acc;
    }
    total[0] = base;
    for (int c = 0; c < nc; c++)
      total[c + 1] += total[c];
#pragma omp parallel for schedule(static)
    for (int c = 0; c < nc; c++) {
      int acc = total[c];
      for (int p = c * kScanChunk; p < std::min(n, (c + 1) * kScanChunk); p++) {
        acc += eai[p + 1];
        eai[p + 1] = acc;
      }
    }
  }
  // rows in execution order, copied on the host's threads
#pragma omp parallel for schedule(dynamic, 4096)
  for (int p = 0; p < n; p++) {
    const int i = erow[p];
    ediag[p] = diag ? diag[i] : 1.0;
    for (int k = ai[i] - base, w = eai[p] - base; k < ai[i + 1] - base; k++, w++) {
      eaj[w] = aj[k];
      eav[w] = av[k];
    }
  }
  P->kd = longest <= 4 ? 4 : longest <= 8 ? 8 : longest <= 16 ? 16 : 0;
  for (int l = 0; l < P->levels; l++)
    for (int p = P->h_prefix[l]; p < P->h_prefix[l + 1]; p += kChunk)
      cstart.push_back(p);
  cstart.push_back(n);
  P->nchunks = (int)cstart.size() - 1;
  LA_TRY(P->ai.upload(eai.get(), sizeof(int) * (n + 1)));
  LA_TRY(P->aj.upload(eaj.get(), sizeof(int) * std::max(P->nnz, 1)));
  LA_TRY(P->exec_row.upload(erow.get(), sizeof(int) * n));
  LA_TRY(P->chunk_start.upload(cstart.data(), sizeof(int) * cstart.size()));
  if (P->dtype == LA_F64) {
    LA_TRY(P->av.upload(eav.get(), sizeof(double) * std::max(P->nnz, 1)));
    LA_TRY(P->diag.upload(ediag.get(), sizeof(double) * n));
    P->grid = grid_for<double, double>(P->nchunks, P->kd);
  } else {
    std::vector<float> f(eav.get(), eav.get() + std::max(P->nnz, 1)),
        fd(ediag.get(), ediag.get() + n);
    LA_TRY(P->av.upload(f.data(), sizeof(float) * f.size()));
    LA_TRY(P->diag.upload(fd.data(), sizeof(float) * n));
    P->grid = grid_for<float, float>(P->nchunks, P->kd);
  }
  return LA_OK;
}

// Reads (and clears) the plan's sticky timeout word; synchronises `st`.
la_status trsv_check(la_trsv_plan_t P, cudaStream_t st) {
  if (P->n == 0)
    return LA_OK;
  int h = 0;
  LA_CUDA_TRY(cudaMemcpyAsync(&h, P->err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  LA_CUDA_TRY(cudaStreamSynchronize(st));
  if (h) {
    LA_CUDA_TRY(cudaMemsetAsync(P->err.p, 0, sizeof(int), st));
    set_error("triangular solve: a dependency wait exceeded its 1 s bound");
    return LA_ERR_TIMEOUT;
  }
  return LA_OK;
}

} // namespace la
