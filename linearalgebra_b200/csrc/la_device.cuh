// la_device.cuh -- device helpers shared by the kernels.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace la {
namespace dev {

// Streaming loads for matrix data read once per call: non-coherent path,
// no L1 allocation (x and y keep the L1/L2 room).
__device__ __forceinline__ int4 ld_stream(const int4 *p) {
  int4 r;
  asm("ld.global.nc.L1::no_allocate.v4.s32 {%0,%1,%2,%3}, [%4];"
      : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
      : "l"(p));
  return r;
}
__device__ __forceinline__ double2 ld_stream(const double2 *p) {
  double2 r;
  asm("ld.global.nc.L1::no_allocate.v2.f64 {%0,%1}, [%2];"
      : "=d"(r.x), "=d"(r.y)
      : "l"(p));
  return r;
}
__device__ __forceinline__ float4 ld_stream(const float4 *p) {
  float4 r;
  asm("ld.global.nc.L1::no_allocate.v4.f32 {%0,%1,%2,%3}, [%4];"
      : "=f"(r.x), "=f"(r.y), "=f"(r.z), "=f"(r.w)
      : "l"(p));
  return r;
}
template <typename T> __device__ __forceinline__ T ld_stream(const T *p) {
  return __ldg(p);
}

// Read-only loads that stay where they are written (asm volatile): used to
// fetch data several steps ahead of its use, which the compiler might
// otherwise move next to the use.
__device__ __forceinline__ int ld_ahead(const int *p) {
  int v;
  asm volatile("ld.global.nc.s32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ float ld_ahead(const float *p) {
  float v;
  asm volatile("ld.global.nc.f32 %0, [%1];" : "=f"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ double ld_ahead(const double *p) {
  double v;
  asm volatile("ld.global.nc.f64 %0, [%1];" : "=d"(v) : "l"(p));
  return v;
}
// 16-byte records (32 for FP64 values), same placement rule
__device__ __forceinline__ int4 ld_ahead(const int4 *p) {
  int4 v;
  asm volatile("ld.global.nc.v4.s32 {%0,%1,%2,%3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "l"(p));
  return v;
}
__device__ __forceinline__ void ld_ahead4(const float *p, float (&v)[4]) {
  asm volatile("ld.global.nc.v4.f32 {%0,%1,%2,%3}, [%4];"
               : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3])
               : "l"(p));
}
__device__ __forceinline__ void ld_ahead4(const double *p, double (&v)[4]) {
  asm volatile("ld.global.nc.v2.f64 {%0,%1}, [%2];" : "=d"(v[0]), "=d"(v[1]) : "l"(p));
  asm volatile("ld.global.nc.v2.f64 {%0,%1}, [%2];" : "=d"(v[2]), "=d"(v[3]) : "l"(p + 2));
}

// Device-scope relaxed accesses (bypass the non-coherent L1) used for data
// exchanged between CTAs of one kernel.
__device__ __forceinline__ double ld_relaxed(const double *p) {
  double v;
  asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ float ld_relaxed(const float *p) {
  float v;
  asm volatile("ld.relaxed.gpu.global.f32 %0, [%1];" : "=f"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed(double *p, double v) {
  asm volatile("st.relaxed.gpu.global.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed(float *p, float v) {
  asm volatile("st.relaxed.gpu.global.f32 [%0], %1;" ::"l"(p), "f"(v) : "memory");
}
__device__ __forceinline__ int ld_relaxed(const int *p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Grid-wide barrier for a cooperative launch.  bar[0]: arrivals, bar[1]:
// generation, bar[2]: error word, set to 1 when a wait gave up after 1 s
// (the waiting block then carries on; callers that loop over barriers read
// bar[2] after each one and leave).  The fences on both sides make the
// writes before the barrier visible to every block after it.
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}
__device__ inline void grid_barrier(unsigned *bar) {
  constexpr unsigned long long kLimitNs = 1000000000ull;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned *gen = bar + 1;
    const unsigned g = *gen; // read before arriving: the generation to leave
    __threadfence();
    if (atomicAdd(bar, 1u) == gridDim.x - 1) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      const unsigned long long t0 = global_ns();
      while (*gen == g) {
        if (global_ns() - t0 > kLimitNs) {
          atomicExch(bar + 2, 1u);
          break;
        }
        __nanosleep(32);
      }
    }
    __threadfence();
  }
  __syncthreads();
}

// Asynchronous 4- or 8-byte copy global -> shared (one element; both
// addresses aligned to its size), tracked by the issuing thread's groups.
template <typename T>
__device__ __forceinline__ void cp_async_shared(T *dst_shared, const T *src) {
  static_assert(sizeof(T) == 4 || sizeof(T) == 8, "cp.async element size");
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst_shared);
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(d), "l"(src),
               "n"(sizeof(T))
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
// every committed group but the most recent one has landed
__device__ __forceinline__ void cp_async_wait_all_but_one() {
  asm volatile("cp.async.wait_group 1;" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_group 0;" ::: "memory");
}

// Segmented-sum pair: f = "a segment boundary occurred", v = running sum
// since the last boundary.  combine(a, b) = (a.f | b.f, b.f ? b.v : a.v+b.v).
template <typename ACC> struct SegPair {
  int f;
  ACC v;
};

// Inclusive warp-level segmented scan.
template <typename ACC>
__device__ __forceinline__ SegPair<ACC> warp_seg_scan_incl(SegPair<ACC> a) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const int f = __shfl_up_sync(0xffffffffu, a.f, d);
    const ACC v = __shfl_up_sync(0xffffffffu, a.v, d);
    if (lane >= d) {
      if (!a.f)
        a.v = v + a.v;
      a.f |= f;
    }
  }
  return a;
}

} // namespace dev
} // namespace la
