// la_trsv.cu -- level-scheduled sparse triangular solve, one persistent
// kernel per solve.
//
// Reference: OptimizedTriangularSolve<Barrier, L|U> (sparse_mat_op/
// triangle_solve.hpp:149-208, triangle_solve.tpp:17-155).  analysis()
// computes level sets with TopologicalSort2 (matrix_utils.hpp:637-675),
// splits every level over the threads and stores the rows physically in
// execution order (permuteRow); the apply walks the levels with an OpenMP
// barrier after each one and computes
//   x[i] = diag ? (b[i] - sum_j T_ij x[j]) / diag[i] : b[i] - sum_j T_ij x[j].
//
// B200 design.  The same host analysis (bit-identical level sets) stores
// the rows in level order and cuts every level into 32-row chunks, so a
// chunk never straddles a level.  One launch of a persistent grid walks all
// levels: warps claim chunks in order from an atomic ticket, one lane per
// row.  Instead of a grid barrier per level, each lane waits only for the x
// entries its row reads: x is pre-filled with a sentinel NaN bit pattern and
// a finished row publishes x[i] with a device-scope store, so a dependency
// is ready when its x entry stops being the sentinel (the value is its own
// flag; one L2 round trip).  Because chunks are claimed in level order, the
// lowest unfinished chunk always has its inputs ready and the solve cannot
// deadlock.  Waiting lanes back off with nanosleep; every wait is bounded by
// the global timer, and on expiry the kernel records a timeout in the plan's
// error word and all warps leave.
//
// Roofline: latency-bound at these sizes (one dependent L2 round trip per
// level); algorithmic bytes per solve
//   nnz*(sizeof(V)+4) + (n+1)*4 + n*4 [exec->row map] + n*sizeof(V) [diag]
//   + n*sizeof(X) [b] + n*sizeof(X) [x].

#include "la_device.cuh"
#include "la_internal.h"

#include <algorithm>
#include <cstdlib>
#include <cstring>

namespace la {
namespace {

constexpr int kThreads = 256;
constexpr int kChunk = 32;
constexpr int kDeps = 8; // dependency loads issued together per row
constexpr unsigned long long kWaitNs = 1000000000ull; // 1 s per wait

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
    }
  }
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
                                                      x, P->base, err, tk);
    break;
  case 8:
    trsv_level_kernel<V, X, UNIT, 8><<<g, t, 0, st>>>(P->nchunks, cs, ai, aj, av, dg, er, b,
                                                      x, P->base, err, tk);
    break;
  case 16:
    trsv_level_kernel<V, X, UNIT, 16><<<g, t, 0, st>>>(P->nchunks, cs, ai, aj, av, dg, er,
                                                       b, x, P->base, err, tk);
    break;
  default:
    trsv_level_kernel_grouped<V, X, UNIT><<<g, t, 0, st>>>(P->nchunks, cs, ai, aj, av, dg,
                                                           er, b, x, P->base, err, tk);
  }
}

template <typename V, typename X>
la_status launch_typed(la_trsv_plan_t P, const X *b, X *x, cudaStream_t st) {
  if (P->n == 0)
    return LA_OK;
  LA_CUDA_TRY(cudaMemsetAsync(x, 0xff, sizeof(X) * (size_t)P->n, st));
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
    P->levels = n == 0 ? 0
                       : topological_sort2(P->uplo, n, base, ai, aj,
                                           P->h_iperm.data(), P->h_prefix.data());
    P->h_prefix.resize(P->levels + 1);
  }
  if (n == 0)
    return LA_OK;
  std::vector<int> eai(n + 1), erow(n), cstart;
  std::vector<int> eaj(std::max(P->nnz, 1));
  std::vector<double> eav(std::max(P->nnz, 1)), ediag(n, 1.0);
  eai[0] = base;
  int w = 0;
  for (int p = 0; p < n; p++) {
    const int i = P->h_iperm[p] - base;
    erow[p] = i;
    if (diag)
      ediag[p] = diag[i];
    for (int k = ai[i] - base; k < ai[i + 1] - base; k++, w++) {
      eaj[w] = aj[k];
      eav[w] = av[k];
    }
    eai[p + 1] = w + base;
  }
  int longest = 0;
  for (int p = 0; p < n; p++)
    longest = std::max(longest, eai[p + 1] - eai[p]);
  P->kd = longest <= 4 ? 4 : longest <= 8 ? 8 : longest <= 16 ? 16 : 0;
  for (int l = 0; l < P->levels; l++)
    for (int p = P->h_prefix[l]; p < P->h_prefix[l + 1]; p += kChunk)
      cstart.push_back(p);
  cstart.push_back(n);
  P->nchunks = (int)cstart.size() - 1;
  LA_TRY(P->ai.upload(eai.data(), sizeof(int) * eai.size()));
  LA_TRY(P->aj.upload(eaj.data(), sizeof(int) * eaj.size()));
  LA_TRY(P->exec_row.upload(erow.data(), sizeof(int) * erow.size()));
  LA_TRY(P->chunk_start.upload(cstart.data(), sizeof(int) * cstart.size()));
  if (P->dtype == LA_F64) {
    LA_TRY(P->av.upload(eav.data(), sizeof(double) * eav.size()));
    LA_TRY(P->diag.upload(ediag.data(), sizeof(double) * n));
    P->grid = grid_for<double, double>(P->nchunks, P->kd);
  } else {
    std::vector<float> f(eav.begin(), eav.end()), fd(ediag.begin(), ediag.end());
    LA_TRY(P->av.upload(f.data(), sizeof(float) * f.size()));
    LA_TRY(P->diag.upload(fd.data(), sizeof(float) * n));
    P->grid = grid_for<float, float>(P->nchunks, P->kd);
  }
  LA_TRY(P->err.alloc(sizeof(int)));
  LA_CUDA_TRY(cudaMemset(P->err.p, 0, sizeof(int)));
  LA_TRY(P->ticket.alloc(sizeof(int)));
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
