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
// chunk never straddles a level.  One cooperative launch keeps every warp
// resident; warp w takes chunks w, w + W, ... in order, one lane per row.
// Instead of a grid barrier per level, each lane waits only for the x
// entries its row reads: x is pre-filled with a sentinel NaN bit pattern and
// a finished row publishes x[i] with a device-scope store, so a dependency
// is ready when its x entry stops being the sentinel (the value is its own
// flag; one L2 round trip).  Chunks are taken in level order, so the lowest
// unfinished chunk always has its inputs ready: the solve cannot deadlock
// while all warps are resident, which the cooperative launch guarantees.
// Every wait is bounded by the global timer; on expiry the kernel records a
// timeout in the plan's error word and all warps leave.
//
// Roofline: latency-bound at these sizes (one dependent L2 round trip per
// level); algorithmic bytes per solve
//   nnz*(sizeof(V)+4) + (n+1)*4 + n*4 [exec->row map] + n*sizeof(V) [diag]
//   + n*sizeof(X) [b] + n*sizeof(X) [x].

#include "la_device.cuh"
#include "la_internal.h"

#include <algorithm>
#include <cstring>

namespace la {
namespace {

constexpr int kThreads = 256;
constexpr int kChunk = 32;
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

template <typename V, typename X, bool UNIT>
__global__ void __launch_bounds__(kThreads)
    trsv_level_kernel(const int nchunks, const int *__restrict__ chunk_start,
                      const int *__restrict__ ai, const int *__restrict__ aj,
                      const V *__restrict__ av, const V *__restrict__ diag,
                      const int *__restrict__ exec_row,
                      const X *__restrict__ b, X *x, const int base, int *err) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * kThreads + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * kThreads) >> 5;
  for (int c = warp; c < nchunks; c += nwarps) {
    const int p = __ldg(chunk_start + c) + lane;
    if (p >= __ldg(chunk_start + c + 1))
      continue;
    const int i = __ldg(exec_row + p);
    X sum = X(0);
    const int ke = __ldg(ai + p + 1) - base;
    for (int k = __ldg(ai + p) - base; k < ke; k++) {
      const int j = __ldg(aj + k) - base;
      X xv = dev::ld_relaxed(x + j);
      if (Sentinel<X>::is(xv)) {
        const unsigned long long t0 = global_ns();
        unsigned polls = 0;
        do {
          if ((++polls & 63u) == 0u) {
            if (dev::ld_relaxed(err) != 0)
              return;
            if (global_ns() - t0 > kWaitNs) {
              atomicExch(err, 1);
              return;
            }
          }
          xv = dev::ld_relaxed(x + j);
        } while (Sentinel<X>::is(xv));
      }
      sum += X(__ldg(av + k)) * xv;
    }
    X xi = __ldg(b + i) - sum;
    if (!UNIT)
      xi = xi / X(__ldg(diag + p));
    dev::st_relaxed(x + i, Sentinel<X>::scrub(xi));
  }
}

template <typename V, typename X>
la_status launch_typed(la_trsv_plan_t P, const X *b, X *x, cudaStream_t st) {
  if (P->n == 0)
    return LA_OK;
  LA_CUDA_TRY(cudaMemsetAsync(x, 0xff, sizeof(X) * (size_t)P->n, st));
  const int *cs = P->chunk_start.as<int>(), *ai = P->ai.as<int>(),
            *aj = P->aj.as<int>(), *er = P->exec_row.as<int>();
  const V *av = P->av.as<V>(), *dg = P->diag.as<V>();
  int *err = P->err.as<int>();
  int nchunks = P->nchunks, base = P->base;
  void *args[] = {&nchunks, &cs, &ai, &aj, &av, &dg, &er, &b, &x, &base, &err};
  const void *fn = P->unit ? (const void *)trsv_level_kernel<V, X, true>
                           : (const void *)trsv_level_kernel<V, X, false>;
  LA_CUDA_TRY(cudaLaunchCooperativeKernel(fn, dim3(P->grid), dim3(kThreads),
                                          args, 0, st));
  return LA_OK;
}

template <typename V, typename X> int grid_for() {
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &per_sm, trsv_level_kernel<V, X, false>, kThreads, 0);
  int per_sm_u = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &per_sm_u, trsv_level_kernel<V, X, true>, kThreads, 0);
  per_sm = std::min(per_sm, per_sm_u);
  return std::max(1, per_sm) * sm_count();
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
la_status trsv_build(la_trsv_plan_t P, const int *ai, const int *aj,
                     const double *av, const double *diag) {
  const int n = P->n, base = P->base;
  P->h_iperm.resize(n);
  P->h_prefix.resize(n + 1);
  P->levels = n == 0 ? 0
                     : topological_sort2(P->uplo, n, base, ai, aj,
                                         P->h_iperm.data(), P->h_prefix.data());
  P->h_prefix.resize(P->levels + 1);
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
    P->grid = grid_for<double, double>();
  } else {
    std::vector<float> f(eav.begin(), eav.end()), fd(ediag.begin(), ediag.end());
    LA_TRY(P->av.upload(f.data(), sizeof(float) * f.size()));
    LA_TRY(P->diag.upload(fd.data(), sizeof(float) * n));
    P->grid = grid_for<float, float>();
  }
  LA_TRY(P->err.alloc(sizeof(int)));
  LA_CUDA_TRY(cudaMemset(P->err.p, 0, sizeof(int)));
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
