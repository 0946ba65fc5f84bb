// la_levels.cu -- level sets of a triangle on the GPU.
//
// Reference: TopologicalSort2<L|U> (sparse_mat_op/matrix_utils.hpp:637-675):
// depth(i) = max over the stored entries j of row i of depth(j) + 1 (0 for a
// row without entries), rows visited ascending for L and descending for U;
// levels = max depth + 1; iperm lists the rows by (level, ascending row)
// with values i + base; prefix[levels + 1] is zero-based.
//
// B200 design.  The depths are a triangular solve in the (max, +) semiring:
// one persistent launch in which warps claim 32-row chunks in the visiting
// order from an atomic ticket, one lane per row; a lane waits (bounded by
// the global timer) until each row it reads has published its depth, then
// publishes its own.  The lowest unfinished row always has its inputs, so
// the pass cannot deadlock.  The rows are then ordered by a stable radix sort
// on their depth (the input order is ascending rows, so ties stay ascending),
// and the level boundaries are the starts of the depth runs.  Integer work
// only: the outputs equal the host's exactly.
//
// Roofline: latency-bound (levels x one L2 round trip) for the depths; the
// sort is HBM-bound (12 bytes moved per row per 8-bit pass).

#include "la_device.cuh"
#include "la_internal.h"

#include <algorithm>
#include <cstdlib>
#include <vector>

namespace la {
namespace {

constexpr int kThreads = 256;
constexpr unsigned long long kWaitNs = 1000000000ull;
constexpr int kGroup = 8; // dependencies polled together
// pause between polls of unpublished depths: fewer polls leave L2 to the
// rows being published (measured, 128^3 IC(0) factor's L, host arrays in and
// out: median 39 ms and up to 81 ms without a pause, 12.8 / 12.0 / 10.4 /
// 10.0 / 10.5 ms with 32 / 128 / 512 / 1024 / 2048 ns, the slowest of eight
// calls 10.4 ms at 1024; 192^3: 20-21 ms throughout; 96^3 27-point: 19.7 ->
// 14.6 ms)
constexpr int kPollSleepNs = 1024;

__device__ __forceinline__ unsigned long long level_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ int ld_acq(const int *p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// depth[] starts at -1 (unpublished).  state[0]: chunk ticket, state[1]: a
// wait gave up, state[2]: an entry outside the strict triangle was seen.
template <bool UPPER>
__global__ void __launch_bounds__(kThreads)
    depth_kernel(const int n, const int base, const int *__restrict__ ai,
                 const int *__restrict__ aj, int *depth, unsigned *key, int *state,
                 const int sleep_ns) {
  const int lane = threadIdx.x & 31, nchunks = (n + 31) / 32;
  for (;;) {
    int c = 0;
    if (lane == 0) // lane 0 alone decides; the warp leaves together
      c = ld_acq(state + 1) != 0 ? nchunks : atomicAdd(state, 1);
    c = __shfl_sync(0xffffffffu, c, 0);
    if (c >= nchunks)
      return;
    const int k = 32 * c + lane;
    if (k >= n)
      continue;
    const int i = UPPER ? n - 1 - k : k;
    int d = 0;
    bool gave_up = false;
    // the row's dependencies kGroup at a time: their depths loaded together,
    // the unpublished ones re-polled until they arrive
    const int e0 = __ldg(ai + i) - base, e1 = __ldg(ai + i + 1) - base;
    const unsigned long long t0 = level_ns();
    for (int g = e0; g < e1 && !gave_up; g += kGroup) {
      int jj[kGroup];
      unsigned pending = 0;
#pragma unroll
      for (int q = 0; q < kGroup; q++) {
        jj[q] = -1;
        if (g + q < e1) {
          const int j = __ldg(aj + g + q) - base;
          if (UPPER ? j <= i : j >= i) // not a dependency on an earlier row
            atomicExch(state + 2, 1);
          else {
            jj[q] = j;
            pending |= 1u << q;
          }
        }
      }
      for (unsigned pass = 1; pending; pass++) {
        int dq[kGroup];
#pragma unroll
        for (int q = 0; q < kGroup; q++)
          dq[q] = (pending >> q) & 1u ? ld_acq(depth + jj[q]) : -1;
#pragma unroll
        for (int q = 0; q < kGroup; q++)
          if (((pending >> q) & 1u) && dq[q] >= 0) {
            d = max(d, dq[q] + 1);
            pending &= ~(1u << q);
          }
        if (pending && (pass & 63u) == 0u &&
            (ld_acq(state + 1) != 0 || level_ns() - t0 > kWaitNs)) {
          atomicExch(state + 1, 1);
          gave_up = true;
          break;
        }
        if (pending && sleep_ns > 0) // back off: fewer polls crowding L2
          __nanosleep(sleep_ns);
      }
    }
    if (gave_up)
      continue;
    key[i] = (unsigned)d;
    __threadfence();
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(depth + i), "r"(d) : "memory");
  }
}

__global__ void iota_u32(const int n, int *v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    v[i] = i;
}

__global__ void max_kernel(const int n, const int *d, int *out) {
  int m = -1;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    m = max(m, d[i]);
  for (int o = 16; o > 0; o >>= 1)
    m = max(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0)
    atomicMax(out, m);
}

__global__ void add_base_kernel(const int n, const int *pos, const int base, int *out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = pos[i] + base;
}

} // namespace

la_status levels_on_device(int uplo, int n, int base, const int *d_ai, const int *d_aj,
                           DevBuf &order, DevBuf &keys, DevBuf &starts, int *levels,
                           cudaStream_t st) {
  *levels = 0;
  if (n == 0)
    return LA_OK;
  DevBuf depth, state, kh[2], kl[2], kp[2];
  LA_TRY(depth.alloc(sizeof(int) * n));
  LA_TRY(state.alloc(sizeof(int) * 4));
  for (int s = 0; s < 2; s++) {
    LA_TRY(kh[s].alloc(sizeof(unsigned) * n));
    LA_TRY(kl[s].alloc(sizeof(unsigned) * n));
    LA_TRY(kp[s].alloc(sizeof(int) * n));
  }
  LA_CUDA_TRY(cudaMemsetAsync(depth.p, 0xff, sizeof(int) * n, st));
  LA_CUDA_TRY(cudaMemsetAsync(state.p, 0, sizeof(int) * 4, st));
  LA_CUDA_TRY(cudaMemsetAsync(kl[0].p, 0, sizeof(unsigned) * n, st));
  int per_sm = 0;
  const void *fn = uplo == LA_LOWER ? (const void *)depth_kernel<false>
                                    : (const void *)depth_kernel<true>;
  LA_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kThreads, 0));
  per_sm = std::max(per_sm, 1);
  if (const char *e = std::getenv("LA_LEVELS_CTAS_PER_SM")) // tuning override
    per_sm = std::min(per_sm, std::max(1, std::atoi(e)));
  const int need = ((n + 31) / 32 + kThreads / 32 - 1) / (kThreads / 32);
  const int grid = std::max(1, std::min(per_sm * sm_count(), need));
  int sleep_ns = kPollSleepNs;
  if (const char *e = std::getenv("LA_LEVELS_SLEEP_NS")) // tuning override
    sleep_ns = std::max(0, std::atoi(e));
  if (uplo == LA_LOWER)
    depth_kernel<false><<<grid, kThreads, 0, st>>>(n, base, d_ai, d_aj, depth.as<int>(),
                                                   kh[0].as<unsigned>(), state.as<int>(),
                                                   sleep_ns);
  else
    depth_kernel<true><<<grid, kThreads, 0, st>>>(n, base, d_ai, d_aj, depth.as<int>(),
                                                  kh[0].as<unsigned>(), state.as<int>(),
                                                  sleep_ns);
  LA_CUDA_TRY(cudaGetLastError());
  const int g = std::max(1, std::min((n + 255) / 256, 8 * sm_count()));
  max_kernel<<<g, 256, 0, st>>>(n, depth.as<int>(), state.as<int>() + 3);
  iota_u32<<<g, 256, 0, st>>>(n, kp[0].as<int>());
  LA_CUDA_TRY(cudaGetLastError());
  int hs[4];
  LA_CUDA_TRY(cudaMemcpyAsync(hs, state.p, sizeof(hs), cudaMemcpyDeviceToHost, st));
  LA_CUDA_TRY(cudaStreamSynchronize(st));
  if (hs[1]) {
    set_error("TopologicalSort2: a dependency wait exceeded its 1 s bound");
    return LA_ERR_TIMEOUT;
  }
  if (hs[2]) {
    set_error("TopologicalSort2: an entry lies outside the strict triangle");
    return LA_ERR_INVALID_ARG;
  }
  const int lv = hs[3] + 1;
  int cur = 0;
  LA_TRY(radix_sort_pairs(n, (unsigned)lv, 1u, kh, kl, kp, &cur, st));
  LA_TRY(starts.alloc(sizeof(int) * (lv + 1)));
  LA_TRY(run_starts(n, kh[cur].as<unsigned>(), lv, 0, starts.as<int>(), st));
  std::swap(order.p, kp[cur].p);
  std::swap(order.bytes, kp[cur].bytes);
  std::swap(keys.p, kh[cur].p);
  std::swap(keys.bytes, kh[cur].bytes);
  LA_CUDA_TRY(cudaStreamSynchronize(st)); // the sort's scratch is released on return
  *levels = lv;
  return LA_OK;
}

la_status topological_sort2_device(int uplo, int n, int base, const int *ai, const int *aj,
                                   int *iperm, int *prefix, int *levels) {
  *levels = 0;
  if (n == 0)
    return LA_OK;
  const int nnz = ai[n] - base;
  cudaStream_t st = nullptr;
  DevBuf dai, daj, order, keys, starts, out;
  LA_TRY(dai.upload(ai, sizeof(int) * (n + 1)));
  LA_TRY(daj.upload(aj, sizeof(int) * std::max(nnz, 1)));
  int lv = 0;
  LA_TRY(levels_on_device(uplo, n, base, dai.as<int>(), daj.as<int>(), order, keys, starts, &lv,
                          st));
  LA_TRY(out.alloc(sizeof(int) * n));
  const int g = std::max(1, std::min((n + 255) / 256, 8 * sm_count()));
  add_base_kernel<<<g, 256, 0, st>>>(n, order.as<int>(), base, out.as<int>());
  LA_CUDA_TRY(cudaGetLastError());
  LA_CUDA_TRY(cudaMemcpyAsync(iperm, out.p, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
  LA_CUDA_TRY(cudaMemcpyAsync(prefix, starts.p, sizeof(int) * (lv + 1), cudaMemcpyDeviceToHost,
                              st));
  LA_CUDA_TRY(cudaStreamSynchronize(st));
  *levels = lv;
  return LA_OK;
}

} // namespace la
