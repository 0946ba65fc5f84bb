// la_spmv.cu -- CSR SpMV on B200 in the reference's two nnz-balanced forms.
//
// Reference: sparse_mat_op/spmv.hpp.  Both reference forms split the
// nonzeros, not the rows, evenly over workers, so long rows never serialise
// on one worker:
//   SegSumSPMV (spmv.hpp:59-185): per-nonzero products alpha*av*b, a
//     segmented inclusive scan inside each chunk, a scan over the chunk
//     carries and a fix-up of each chunk's leading open segment;
//   ALBUSSPMV (spmv.hpp:186-300): per-chunk sums of the partial first row,
//     the whole interior rows and the partial last row, merged afterwards.
//
// B200 design.  A "tile" is kTile = 1024 consecutive nonzeros, one CTA of
// 256 threads; the plan stores the row that holds each tile's first nonzero
// (the reference's ALBUS preprocess, spmv.hpp:210-217), so a tile is the
// GPU's counterpart of one reference worker's chunk.  Small tiles and small
// per-thread work keep many CTAs resident, which is what hides the HBM and
// gather latency here.  In a tile:
//  1. every thread streams 4 column indices and 4 values (warp-coalesced,
//     non-allocating loads), gathers x through the read-only path (x of
//     every configuration here fits in the 126 MB L2) as soon as its columns
//     land, stages the tile's row pointers in shared memory and writes the
//     products there;
//  2. one thread per row sums that row's products in column order with
//     exact (never fused) multiplies and adds, so every row that lies inside
//     a tile is bit-identical to the reference's sequential loop; in-tile
//     segments longer than 64 are summed by a warp;
//  3. complete rows are written; a row that crosses a tile edge leaves a
//     head / tail partial per tile, as the reference's boundary values do
//     (spmv.hpp:244-264).
// A second kernel, launched with programmatic dependent launch so that its
// start overlaps the first one's tail, finalises each crossing row by adding
// its partials in tile order -- the reference's merge order.  No fence, no
// atomic and no spin-wait is involved; the result is deterministic.
//
// Roofline: HBM-bound.  Algorithmic bytes per call
//   nnz*(sizeof(V) + 4) + (n+1)*4 + n*sizeof(X) [x] + n*sizeof(X) [y]
//   (+ n*sizeof(X) when beta != 0).

#include "la_device.cuh"
#include "la_internal.h"

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <type_traits>

namespace la {
namespace {

constexpr int kThreads = 256;
constexpr int kTileBlocksPerSm = 8;      // tile pass: 8 x 256 threads per SM
constexpr int kNpt = 4;                  // nonzeros per thread
constexpr int kTile = kThreads * kNpt;   // nonzeros per tile
constexpr int kRowCap = kTile + 1;       // staged row pointers per tile
constexpr int kLongRow = 64;             // in-tile segments longer than this
                                         // are summed by a warp
constexpr int kLongCap = kTile / (kLongRow + 1) + 2;
constexpr int kVecRow = 8;               // 16-byte loads when no row is longer

enum Form { kSegSum = 0, kAlbus = 1 };

// Exact IEEE operations: never fused into an FMA, so a row summed by one
// thread reproduces the reference's `val += av[j] * b[aj[j]]` bit for bit.
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }

// Matrix data is read once per call: non-coherent path, no L1 allocation.
__device__ __forceinline__ double ld_once(const double *p) {
  double v;
  asm("ld.global.nc.L1::no_allocate.f64 %0, [%1];" : "=d"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ float ld_once(const float *p) {
  float v;
  asm("ld.global.nc.L1::no_allocate.f32 %0, [%1];" : "=f"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ int ld_once(const int *p) {
  int v;
  asm("ld.global.nc.L1::no_allocate.s32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}

template <int FORM, typename ACC> struct RowOut {
  ACC alpha, beta;
  // A whole row finished inside one tile:
  //   ALBUS / Serial (spmv.hpp:256):  alpha * val + (beta == 0 ? 0 : beta * x)
  //   SegSum (spmv.hpp:171):          val + beta * x   (val already scaled)
  // beta == 0 never reads y.
  template <typename X>
  __device__ __forceinline__ void write(X *y, const X *yin, int r, ACC sum) const {
    const ACC v = FORM == kAlbus ? mul_rn(alpha, sum) : sum;
    y[r] = X(beta == ACC(0) ? v : add_rn(v, mul_rn(beta, ACC(yin[r]))));
  }
  // A partial row handed to the merge (ALBUS scales partials).
  __device__ __forceinline__ ACC partial(ACC sum) const {
    return FORM == kAlbus ? mul_rn(alpha, sum) : sum;
  }
};

// A tile's nonzero range [s, s + cnt) and row span [R0, Rlast]; R1 is the
// row holding the next tile's first nonzero (n after the last tile).
struct TileRows {
  int s, cnt, R0, R1, Rlast, nrows;
  bool staged;
};

__device__ __forceinline__ TileRows tile_rows(int t, int n, int nnz,
                                              const int *__restrict__ tile_row) {
  TileRows T;
  T.s = t * kTile;
  T.cnt = min(T.s + kTile, nnz) - T.s;
  T.R0 = __ldg(tile_row + t);
  T.R1 = __ldg(tile_row + t + 1);
  T.Rlast = min(T.R1, n - 1);
  T.nrows = T.Rlast - T.R0 + 1;
  T.staged = T.nrows + 1 <= kRowCap;
  return T;
}

// Tile-local start of row R0 + i, clamped to [0, cnt]; staged in shared
// memory when the tile's row span fits (it always does without empty rows).
__device__ __forceinline__ void stage_rows(const TileRows &T, int base,
                                           const int *__restrict__ ai, int *rp) {
  if (T.staged)
    for (int i = threadIdx.x; i <= T.nrows; i += kThreads)
      rp[i] = min(max(__ldg(ai + T.R0 + i) - base - T.s, 0), T.cnt);
}

__device__ __forceinline__ int row_start(const TileRows &T, int base,
                                         const int *__restrict__ ai,
                                         const int *rp, int i) {
  return T.staged ? rp[i] : min(max(__ldg(ai + T.R0 + i) - base - T.s, 0), T.cnt);
}

// x split into contiguous slices (la_spmv_xparts): slice r holds columns
// [start[r], start[r+1]) at p[r], which may be another GPU's memory.
template <typename X> struct XParts {
  const X *p[LA_SPMV_MAX_XPARTS];
  int start[LA_SPMV_MAX_XPARTS + 1];
  int n;
};

// 16-byte vector loads of a full tile's columns and values for VEC tiles:
// thread tid owns nonzeros [4 tid, 4 tid + 4) of the tile.
__device__ __forceinline__ void ld_vec4(const int *p, int (&j)[kNpt]) {
  asm("ld.global.nc.L1::no_allocate.v4.s32 {%0,%1,%2,%3}, [%4];"
      : "=r"(j[0]), "=r"(j[1]), "=r"(j[2]), "=r"(j[3])
      : "l"(p));
}
__device__ __forceinline__ void ld_vec4(const double *p, double (&v)[kNpt]) {
  asm("ld.global.nc.L1::no_allocate.v2.f64 {%0,%1}, [%2];" : "=d"(v[0]), "=d"(v[1]) : "l"(p));
  asm("ld.global.nc.L1::no_allocate.v2.f64 {%0,%1}, [%2];"
      : "=d"(v[2]), "=d"(v[3])
      : "l"(p + 2));
}
__device__ __forceinline__ void ld_vec4(const float *p, float (&v)[kNpt]) {
  asm("ld.global.nc.L1::no_allocate.v4.f32 {%0,%1,%2,%3}, [%4];"
      : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3])
      : "l"(p));
}
__device__ __forceinline__ void st_vec4(double *p, const double (&v)[kNpt]) {
  *reinterpret_cast<double2 *>(p) = make_double2(v[0], v[1]);
  *reinterpret_cast<double2 *>(p + 2) = make_double2(v[2], v[3]);
}
__device__ __forceinline__ void st_vec4(float *p, const float (&v)[kNpt]) {
  *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
}

// Tile pass of y = alpha*A*x + beta*yin (yin may equal y).  With XP the
// gather reads column j from the slice that owns it (XParts) instead of x.
// LONG = false drops the warp path for in-tile segments longer than kLongRow
// (and its second barrier); the plan selects it when no row is that long.
// CHUNK: the grid covers tiles [tile0, tile0 + grid) (chunked host-pointer
// calls); otherwise tile0 is not read, which keeps the kernel's schedule.
// VEC: a full tile's columns and values are read with 16-byte loads, thread
// tid owning its 4 consecutive nonzeros, instead of one element per 256-wide
// stride.  Same products, same row sums: the results are bit-identical.  The
// plan selects it when no row has more than kVecRow entries (measured on the
// 128^3 Laplacian: 44.1 against 45.1 us back to back, 52.2 against 56.3 us
// with L2 flushed); with the 27-entry rows of the 96^3 stencil's transpose
// it measured slower (78.8 against 71.3 us), as on the power-law matrix,
// whose rows reach 20000 entries (186.6 against 178.1 us).  It needs 16-byte
// aligned aj / av, which the plan's own copies are.
template <int FORM, typename V, typename X, typename ACC, bool XP = false, bool LONG = true,
          bool CHUNK = false, bool VEC = false>
__global__ void __launch_bounds__(kThreads, kTileBlocksPerSm)
    spmv_tile_kernel(const int n, const int nnz, const int base,
                     const int *__restrict__ ai, const int *__restrict__ aj,
                     const V *__restrict__ av, const X *__restrict__ x, X *y,
                     const X *yin, const ACC alpha, const ACC beta,
                     const int *__restrict__ tile_row, ACC *part,
                     const XParts<X> xp = XParts<X>{}, const int tile0 = 0) {
  __shared__ __align__(16) ACC prod[kTile];
  __shared__ int rp[kRowCap];
  __shared__ int long_rows[kLongCap];
  __shared__ int n_long;
  __shared__ const X *xp_ptr[XP ? LA_SPMV_MAX_XPARTS : 1];
  __shared__ int xp_start[XP ? LA_SPMV_MAX_XPARTS + 1 : 1];
  if (XP) { // constant indices keep the parameter block out of local memory
    if (threadIdx.x == 0) {
#pragma unroll
      for (int r = 0; r < LA_SPMV_MAX_XPARTS; r++)
        xp_ptr[r] = xp.p[r];
#pragma unroll
      for (int r = 0; r <= LA_SPMV_MAX_XPARTS; r++)
        xp_start[r] = xp.start[r];
    }
    __syncthreads();
  }
  // let the merge kernel's launch overlap this grid
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  const RowOut<FORM, ACC> out{alpha, beta};
  const int t = CHUNK ? blockIdx.x + tile0 : blockIdx.x, tid = threadIdx.x;
  const TileRows T = tile_rows(t, n, nnz, tile_row);
  if (LONG && tid == 0)
    n_long = 0;
  if (t == 0) // leading empty rows (ai[r + 1] == ai[0]) precede tile 0
    for (int r = tid; r < T.R0; r += kThreads)
      out.write(y, yin, r, ACC(0));
  // Load order (measured on the 128^3 Laplacian and the 4M-row power-law
  // matrix): all column indices first and the x gathers as soon as they
  // land, so the gathers' L2 latency overlaps the values' HBM latency.
  // 4-byte values are loaded together with the columns; 8-byte values after
  // the gathers are issued, which keeps the kernel at 32 registers (8 CTAs
  // of 256 threads per SM) without spills.
  constexpr bool kValuesFirst = sizeof(V) == 4;
  const bool full = T.cnt == kTile;
  if (VEC && full) {
    const int k0 = kNpt * tid;
    int jj[kNpt];
    V vv[kNpt];
    ld_vec4(aj + T.s + k0, jj);
    if (kValuesFirst)
      ld_vec4(av + T.s + k0, vv);
    ACC xv[kNpt];
#pragma unroll
    for (int q = 0; q < kNpt; q++)
      xv[q] = ACC(__ldg(x + jj[q] - base));
    if (!kValuesFirst)
      ld_vec4(av + T.s + k0, vv);
    stage_rows(T, base, ai, rp);
    ACC pv[kNpt];
#pragma unroll
    for (int q = 0; q < kNpt; q++) {
      const ACC v = ACC(vv[q]);
      pv[q] = FORM == kSegSum ? mul_rn(mul_rn(alpha, v), xv[q]) : mul_rn(v, xv[q]);
    }
    st_vec4(prod + k0, pv);
  } else {
  int jj[kNpt];
  V vv[kNpt];
#pragma unroll
  for (int q = 0; q < kNpt; q++) {
    const int kk = q * kThreads + tid;
    if (full || kk < T.cnt) {
      jj[q] = ld_once(aj + T.s + kk);
      if (kValuesFirst)
        vv[q] = ld_once(av + T.s + kk);
    }
  }
  ACC xv[kNpt];
#pragma unroll
  for (int q = 0; q < kNpt; q++)
    if (full || q * kThreads + tid < T.cnt) {
      if (XP) { // owner: the number of slice starts at or below the column
        const int j = jj[q] - base;
        int r = 0;
        for (int k = 1; k < xp.n; k++)
          r += j >= xp_start[k];
        xv[q] = ACC(__ldg(xp_ptr[r] + (j - xp_start[r])));
      } else {
        xv[q] = ACC(__ldg(x + jj[q] - base));
      }
    }
  stage_rows(T, base, ai, rp);
#pragma unroll
  for (int q = 0; q < kNpt; q++) {
    const int kk = q * kThreads + tid;
    if (full || kk < T.cnt) {
      const ACC v = ACC(kValuesFirst ? vv[q] : ld_once(av + T.s + kk));
      prod[kk] = FORM == kSegSum ? mul_rn(mul_rn(alpha, v), xv[q]) : mul_rn(v, xv[q]);
    }
  }
  } // !(VEC && full)
  __syncthreads();

  auto emit = [&](int r, ACC sum) {
    if (r == T.R0)
      part[2 * t] = out.partial(sum);
    else if (r == T.R1)
      part[2 * t + 1] = out.partial(sum);
    else
      out.write(y, yin, r, sum);
  };
  for (int i = tid; i < T.nrows; i += kThreads) {
    const int lo = row_start(T, base, ai, rp, i), hi = row_start(T, base, ai, rp, i + 1);
    if (LONG && hi - lo > kLongRow) {
      long_rows[atomicAdd(&n_long, 1)] = i;
      continue;
    }
    ACC sum = ACC(0);
    for (int k = lo; k < hi; k++)
      sum = add_rn(sum, prod[k]);
    emit(T.R0 + i, sum);
  }
  if (!LONG)
    return;
  __syncthreads();
  const int lane = tid & 31, warp = tid >> 5;
  for (int li = warp; li < n_long; li += kThreads / 32) {
    const int i = long_rows[li];
    const int lo = row_start(T, base, ai, rp, i), hi = row_start(T, base, ai, rp, i + 1);
    ACC sum = ACC(0);
    for (int k = lo + lane; k < hi; k += 32)
      sum = add_rn(sum, prod[k]);
#pragma unroll
    for (int d = 16; d > 0; d >>= 1)
      sum = add_rn(sum, __shfl_down_sync(0xffffffffu, sum, d));
    if (lane == 0)
      emit(T.R0 + i, sum);
  }
}

// Merge pass: one thread per tile f that is the first tile holding its head
// row R; adds the previous tile's tail partial and the head partials of
// every tile that starts inside R, in tile order, and writes y[R].  The
// tiles of that group are [f, group_end[f]) (group_end[f] = -1 when f is not
// the first); plan-built groups are constant, so they are read before the
// wait for the tile pass and the partials' loads do not depend on one
// another.  Without group_end (the allocation-free path, whose tile rows are
// computed on the device) the group is found by scanning tile_row.
// After the tile pass over tiles [t0, t1) only (a chunk of a host-pointer
// call), the groups whose last tile lies in that range are merged; threads
// start at f0, the first tile of the group holding tile t0.
template <int FORM, typename X, typename ACC, bool CHUNK = false>
__global__ void __launch_bounds__(256)
    spmv_merge_kernel(const int ntiles, X *y, const X *yin, const ACC beta,
                      const int *__restrict__ tile_row, const ACC *part,
                      const int *__restrict__ group_end, const int f0 = 0, const int t0 = 0,
                      const int t1 = 0) {
  const int f = (CHUNK ? f0 : 0) + blockIdx.x * blockDim.x + threadIdx.x;
  int R = 0, e = -1;
  if (group_end && f < ntiles) {
    e = group_end[f];
    if (CHUNK && (e - 1 < t0 || e - 1 >= t1)) // a head whose group ends elsewhere
      e = -1;
    if (e >= 0)
      R = tile_row[f];
  }
  // wait until the tile pass has completed and its writes are visible
  asm volatile("griddepcontrol.wait;" ::: "memory");
  if (f >= ntiles)
    return;
  if (!group_end) {
    R = tile_row[f];
    if (f > 0 && tile_row[f - 1] == R)
      return;
    e = f + 1;
    while (e < ntiles && tile_row[e] == R)
      e++;
  }
  if (e < 0)
    return;
  if (FORM == kAlbus) { // merge order of spmv.hpp:275-292
    ACC v = beta == ACC(0) ? ACC(0) : mul_rn(beta, ACC(yin[R]));
    if (f > 0)
      v = add_rn(v, part[2 * (f - 1) + 1]);
#pragma unroll 4
    for (int u = f; u < e; u++)
      v = add_rn(v, part[2 * u]);
    y[R] = X(v);
  } else { // carry chain of spmv.hpp:118-141, then + beta*x (:171)
    ACC c = f > 0 ? part[2 * (f - 1) + 1] : ACC(0);
#pragma unroll 4
    for (int u = f; u < e; u++)
      c = add_rn(part[2 * u], c);
    y[R] = X(beta == ACC(0) ? c : add_rn(c, mul_rn(beta, ACC(yin[R]))));
  }
}

// nnz == 0: every row is empty.
template <typename X, typename ACC>
__global__ void spmv_empty_kernel(int n, X *y, const X *yin, ACC beta) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n;
       r += gridDim.x * blockDim.x)
    y[r] = X(beta == ACC(0) ? ACC(0) : beta * ACC(yin[r]));
}

// dv[k] = alpha * g[row(k)] * x[col(k)] over the stored pattern.  The column
// loads and x gathers are issued first; meanwhile every nonempty row of the
// tile marks the slot of its first nonzero with its tile-local index, and an
// inclusive max-scan over the tile's 1024 slots (4 consecutive slots per
// thread, a warp shuffle scan, the warps' totals in shared memory) gives
// every nonzero its row -- the last row starting at or before it -- with no
// search.  A tile whose row span does not fit in shared memory (runs of
// empty rows) finds its rows by binary search in the row pointers.
__global__ void __launch_bounds__(kThreads)
    sddmm_kernel(const int n, const int nnz, const int base,
                 const int *__restrict__ ai, const int *__restrict__ aj,
                 const double *__restrict__ g, const double *__restrict__ x,
                 double *__restrict__ dv, const double alpha,
                 const int *__restrict__ tile_row) {
  __shared__ int rp[kRowCap];
  __shared__ int row_of[kTile];
  __shared__ int wmax[kThreads / 32];
  const TileRows T = tile_rows(blockIdx.x, n, nnz, tile_row);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  int jj[kNpt];
  double xv[kNpt];
#pragma unroll
  for (int q = 0; q < kNpt; q++) {
    const int kk = q * kThreads + tid;
    if (kk < T.cnt)
      jj[q] = ld_once(aj + T.s + kk);
  }
#pragma unroll
  for (int q = 0; q < kNpt; q++)
    if (q * kThreads + tid < T.cnt)
      xv[q] = __ldg(x + jj[q] - base);
  stage_rows(T, base, ai, rp);
#pragma unroll
  for (int q = 0; q < kNpt; q++)
    row_of[q * kThreads + tid] = -1;
  __syncthreads();
  if (T.staged) {
    for (int i = tid; i < T.nrows; i += kThreads) // distinct starts: nonempty rows
      if (rp[i] < rp[i + 1])
        row_of[rp[i]] = i;
    __syncthreads();
    const int k0 = kNpt * tid;
    int r[kNpt], m = -1;
#pragma unroll
    for (int q = 0; q < kNpt; q++) {
      m = max(m, row_of[k0 + q]);
      r[q] = m;
    }
    int incl = m;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, incl, d);
      if (lane >= d)
        incl = max(incl, v);
    }
    if (lane == 31)
      wmax[warp] = incl;
    int before = __shfl_up_sync(0xffffffffu, incl, 1);
    if (lane == 0)
      before = -1;
    __syncthreads();
    for (int w = 0; w < warp; w++)
      before = max(before, wmax[w]);
#pragma unroll
    for (int q = 0; q < kNpt; q++)
      row_of[k0 + q] = max(before, r[q]);
    __syncthreads();
  } else {
#pragma unroll
    for (int q = 0; q < kNpt; q++) {
      const int kk = q * kThreads + tid;
      if (kk >= T.cnt)
        continue;
      int lo = 0, hi = T.nrows - 1; // last row i with start(i) <= kk
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (row_start(T, base, ai, rp, mid) <= kk)
          lo = mid;
        else
          hi = mid - 1;
      }
      row_of[kk] = lo;
    }
  }
#pragma unroll
  for (int q = 0; q < kNpt; q++) {
    const int kk = q * kThreads + tid;
    if (kk < T.cnt)
      dv[T.s + kk] = alpha * __ldg(g + T.R0 + row_of[kk]) * xv[q];
  }
}

// The achievable bound of a matrix (measurement aid, not an SpMV): every
// CTA streams one tile's columns and values with 16-byte loads and, when
// GATHER, gathers x through the columns -- the SpMV tile pass without its row
// structure (no row pointers, no products in shared memory, no row sums, no
// partials, no merge).  Each thread's sum is kept live by a store that never
// happens unless it equals the unlikely `guard`.
template <bool GATHER>
__global__ void __launch_bounds__(kThreads, kTileBlocksPerSm)
    spmv_ceiling_kernel(const int nnz, const int base, const int *__restrict__ aj,
                        const double *__restrict__ av, const double *__restrict__ x,
                        double *sink, const double guard) {
  const int k0 = blockIdx.x * kTile + kNpt * threadIdx.x;
  if (k0 + kNpt > nnz)
    return;
  int jj[kNpt];
  double vv[kNpt];
  ld_vec4(aj + k0, jj);
  ld_vec4(av + k0, vv);
  double s = 0.0;
#pragma unroll
  for (int q = 0; q < kNpt; q++)
    s += GATHER ? vv[q] * __ldg(x + jj[q] - base) : vv[q] + double(jj[q]);
  if (s == guard)
    sink[0] = s;
}

// ---- Row-slot form for matrices whose rows all hold at most kEllRow
// entries: slot s of row r at s * n + r (column -1 past the row's end), so a
// thread owns a row and every load of a warp is coalesced, with no row
// pointer to read first, no shared memory, no barrier and no merge.  The row
// is summed by its thread in stored order with the same exact operations as
// a row inside one tile of the tile pass (products first, starting from 0):
// y is SerialSPMV's row sum, formed as SegSum / ALBUS form it.
constexpr int kEllRow = 8;
constexpr int kEllMinRows = 65536;

template <int FORM, typename V, typename X, typename ACC>
__global__ void __launch_bounds__(kThreads)
    spmv_ell_kernel(const int n, const int k, const int r0, const int r1,
                    const int *__restrict__ ej, const V *__restrict__ ev,
                    const X *__restrict__ x, X *y, const X *yin, const ACC alpha,
                    const ACC beta) {
  const RowOut<FORM, ACC> out{alpha, beta};
  for (int r = r0 + blockIdx.x * blockDim.x + threadIdx.x; r < r1;
       r += gridDim.x * blockDim.x) {
    int jj[kEllRow];
#pragma unroll
    for (int s = 0; s < kEllRow; s++)
      jj[s] = s < k ? ld_once(ej + (size_t)s * n + r) : -1;
    ACC xv[kEllRow];
#pragma unroll
    for (int s = 0; s < kEllRow; s++)
      xv[s] = jj[s] >= 0 ? ACC(__ldg(x + jj[s])) : ACC(0);
    ACC sum = ACC(0);
#pragma unroll
    for (int s = 0; s < kEllRow; s++)
      if (jj[s] >= 0) {
        const ACC v = ACC(ld_once(ev + (size_t)s * n + r));
        sum = add_rn(sum, FORM == kSegSum ? mul_rn(mul_rn(alpha, v), xv[s]) : mul_rn(v, xv[s]));
      }
    out.write(y, yin, r, sum);
  }
}

template <typename V>
__global__ void ell_build_kernel(const int n, const int k, const int base,
                                 const int *__restrict__ ai, const int *__restrict__ aj,
                                 const V *__restrict__ av, int *ej, V *ev) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const int a = ai[r] - base, len = ai[r + 1] - base - a;
    for (int s = 0; s < k; s++) {
      if (ej)
        ej[(size_t)s * n + r] = s < len ? aj[a + s] - base : -1;
      ev[(size_t)s * n + r] = s < len ? av[a + s] : V(0);
    }
  }
}

template <int FORM, typename V, typename X, typename ACC>
la_status launch_ell(la_spmv_plan_t P, const V *ev, ACC alpha, const X *x, ACC beta, X *y,
                     const X *yin, cudaStream_t st, int r0 = 0, int r1 = -1) {
  const int n = P->A->n;
  if (r1 < 0)
    r1 = n;
  if (r1 <= r0)
    return LA_OK;
  const int g = std::max(1, std::min((r1 - r0 + kThreads - 1) / kThreads, 32 * sm_count()));
  spmv_ell_kernel<FORM, V, X, ACC><<<g, kThreads, 0, st>>>(n, P->ell_k, r0, r1,
                                                            P->ell_j.as<int>(), ev, x, y, yin,
                                                            alpha, beta);
  LA_CUDA_TRY(cudaGetLastError());
  return LA_OK;
}

// Tiles [tile0, tile1) only when tile1 >= 0 (a chunk of a host-pointer call:
// the plan's host copies of tile_row and group_end give the merge range).
template <int FORM, typename V, typename X, typename ACC, bool XP = false>
la_status launch_form(la_spmv_plan_t P, const V *av, ACC alpha, const X *x,
                      ACC beta, X *y, const X *yin, cudaStream_t st,
                      const XParts<X> &xp = XParts<X>{}, int tile0 = 0, int tile1 = -1) {
  const la_csr_t A = P->A;
  if (A->n == 0)
    return LA_OK;
  if (A->nnz == 0) {
    spmv_empty_kernel<X, ACC><<<std::min((A->n + 255) / 256, 4096), 256, 0, st>>>(
        A->n, y, yin, beta);
    LA_CUDA_TRY(cudaGetLastError());
    return LA_OK;
  }
  const bool chunk = tile1 >= 0;
  // short rows only: 16-byte loads (not with x slices, whose gathers keep
  // the element layout)
  auto tile = chunk ? (P->long_rows ? spmv_tile_kernel<FORM, V, X, ACC, XP, true, true>
                      : P->vec_tiles ? spmv_tile_kernel<FORM, V, X, ACC, XP, false, true, !XP>
                                     : spmv_tile_kernel<FORM, V, X, ACC, XP, false, true>)
                    : (P->long_rows ? spmv_tile_kernel<FORM, V, X, ACC, XP, true>
                      : P->vec_tiles ? spmv_tile_kernel<FORM, V, X, ACC, XP, false, false, !XP>
                                     : spmv_tile_kernel<FORM, V, X, ACC, XP, false>);
  if (tile1 < 0)
    tile1 = P->ntiles;
  int f0 = 0;
  if (tile0 > 0)
    for (f0 = tile0; f0 > 0 && P->h_group_end[f0] < 0;)
      f0--;
  tile<<<tile1 - tile0, kThreads, 0, st>>>(A->n, A->nnz, A->base, A->ai.as<int>(),
                                           A->aj.as<int>(), av, x, y, yin, alpha, beta,
                                           P->tile_row.as<int>(), P->part.as<ACC>(), xp,
                                           tile0);
  LA_CUDA_TRY(cudaGetLastError());
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((tile1 - f0 + 255) / 256);
  cfg.blockDim = dim3(256);
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  const int nt = P->ntiles;
  const int *tr = P->tile_row.as<int>();
  const ACC *pt = P->part.as<ACC>();
  const int *ge = P->group_end.as<int>();
  if (chunk)
    LA_CUDA_TRY(cudaLaunchKernelEx(&cfg, spmv_merge_kernel<FORM, X, ACC, true>, nt, y, yin,
                                   beta, tr, pt, ge, f0, tile0, tile1));
  else
    LA_CUDA_TRY(cudaLaunchKernelEx(&cfg, spmv_merge_kernel<FORM, X, ACC>, nt, y, yin, beta,
                                   tr, pt, ge, f0, tile0, tile1));
  return LA_OK;
}

} // namespace

// Internal entry used by the solvers: y = alpha*A*x + beta*yin.
la_status spmv_launch(la_spmv_plan_t P, double alpha, const void *x,
                      double beta, void *y, const void *yin, la_dtype vd,
                      cudaStream_t st) {
  const la_csr_t A = P->A;
  if (vd == LA_F64) {
    if (A->dtype != LA_F64) {
      set_error("FP64 SpMV needs an FP64 matrix");
      return LA_ERR_INVALID_ARG;
    }
    const double *av = A->av.as<double>();
    if (P->ell_k) {
      const double *ev = P->ell_v.as<double>();
      if (P->kind == LA_SPMV_ALBUS)
        return launch_ell<kAlbus>(P, ev, alpha, (const double *)x, beta, (double *)y,
                                  (const double *)yin, st);
      return launch_ell<kSegSum>(P, ev, alpha, (const double *)x, beta, (double *)y,
                                 (const double *)yin, st);
    }
    if (P->kind == LA_SPMV_ALBUS)
      return launch_form<kAlbus>(P, av, alpha, (const double *)x, beta,
                                 (double *)y, (const double *)yin, st);
    return launch_form<kSegSum>(P, av, alpha, (const double *)x, beta,
                                (double *)y, (const double *)yin, st);
  }
  const float *av = static_cast<const float *>(A->values(LA_F32));
  if (!av) {
    set_error("FP32 SpMV needs FP32 values (LA_CSR_KEEP_F32 or an FP32 matrix)");
    return LA_ERR_INVALID_ARG;
  }
  const float fa = (float)alpha, fb = (float)beta;
  if (P->ell_k && P->ell_v32.p) {
    const float *ev = P->ell_v32.as<float>();
    if (P->kind == LA_SPMV_ALBUS)
      return launch_ell<kAlbus>(P, ev, fa, (const float *)x, fb, (float *)y,
                                (const float *)yin, st);
    return launch_ell<kSegSum>(P, ev, fa, (const float *)x, fb, (float *)y,
                               (const float *)yin, st);
  }
  if (P->kind == LA_SPMV_ALBUS)
    return launch_form<kAlbus>(P, av, fa, (const float *)x, fb, (float *)y,
                               (const float *)yin, st);
  return launch_form<kSegSum>(P, av, fa, (const float *)x, fb, (float *)y,
                              (const float *)yin, st);
}

// y = alpha*A*x + beta*y with x given as slices (validated by the caller).
la_status spmv_xparts_launch(la_spmv_plan_t P, double alpha, const void *const *xparts,
                             const int *part_start, int nparts, double beta, void *y,
                             la_dtype vd, cudaStream_t st) {
  auto fill = [&](auto &xp) {
    using X = std::remove_cv_t<std::remove_pointer_t<std::remove_cv_t<
        std::remove_reference_t<decltype(xp.p[0])>>>>;
    for (int r = 0; r < LA_SPMV_MAX_XPARTS; r++)
      xp.p[r] = r < nparts ? static_cast<const X *>(xparts[r]) : nullptr;
    for (int r = 0; r <= LA_SPMV_MAX_XPARTS; r++)
      xp.start[r] = part_start[std::min(r, nparts)];
    xp.n = nparts;
  };
  const la_csr_t A = P->A;
  if (vd == LA_F64) {
    if (A->dtype != LA_F64) {
      set_error("FP64 SpMV needs an FP64 matrix");
      return LA_ERR_INVALID_ARG;
    }
    XParts<double> xp;
    fill(xp);
    const double *av = A->av.as<double>();
    double *yy = static_cast<double *>(y);
    if (P->kind == LA_SPMV_ALBUS)
      return launch_form<kAlbus, double, double, double, true>(P, av, alpha, nullptr, beta, yy,
                                                                yy, st, xp);
    return launch_form<kSegSum, double, double, double, true>(P, av, alpha, nullptr, beta, yy,
                                                               yy, st, xp);
  }
  const float *av = static_cast<const float *>(A->values(LA_F32));
  if (!av) {
    set_error("FP32 SpMV needs FP32 values (LA_CSR_KEEP_F32 or an FP32 matrix)");
    return LA_ERR_INVALID_ARG;
  }
  XParts<float> xp;
  fill(xp);
  float *yy = static_cast<float *>(y);
  if (P->kind == LA_SPMV_ALBUS)
    return launch_form<kAlbus, float, float, float, true>(P, av, (float)alpha, nullptr,
                                                          (float)beta, yy, yy, st, xp);
  return launch_form<kSegSum, float, float, float, true>(P, av, (float)alpha, nullptr,
                                                         (float)beta, yy, yy, st, xp);
}

la_status spmv_ceiling_launch(la_spmv_plan_t P, const double *x, int gather, double *sink,
                              cudaStream_t st) {
  const la_csr_t A = P->A;
  if (A->nnz < kTile || A->dtype != LA_F64) {
    set_error("la_spmv_ceiling: an FP64 matrix of at least %d nonzeros", kTile);
    return LA_ERR_INVALID_ARG;
  }
  const int grid = A->nnz / kTile; // whole tiles only
  if (gather)
    spmv_ceiling_kernel<true><<<grid, kThreads, 0, st>>>(A->nnz, A->base, A->aj.as<int>(),
                                                          A->av.as<double>(), x, sink, 1e300);
  else
    spmv_ceiling_kernel<false><<<grid, kThreads, 0, st>>>(A->nnz, A->base, A->aj.as<int>(),
                                                           A->av.as<double>(), x, sink, 1e300);
  LA_CUDA_TRY(cudaGetLastError());
  return LA_OK;
}

la_status sddmm_launch(la_spmv_plan_t P, double alpha, const double *g,
                       const double *x, double *dv, cudaStream_t st) {
  const la_csr_t A = P->A;
  if (A->nnz == 0)
    return LA_OK;
  sddmm_kernel<<<P->ntiles, kThreads, 0, st>>>(A->n, A->nnz, A->base, A->ai.as<int>(),
                                               A->aj.as<int>(), g, x, dv, alpha,
                                               P->tile_row.as<int>());
  LA_CUDA_TRY(cudaGetLastError());
  return LA_OK;
}

// Plan: the row holding each tile's first nonzero (upper_bound on ai, as
// ALBUSSPMV::preprocess does, spmv.hpp:210-217) and the partial-sum scratch.
la_status spmv_plan_build(la_spmv_plan_t P) {
  const la_csr_t A = P->A;
  const int n = A->n, nnz = A->nnz, base = A->base;
  const int ntiles = nnz == 0 ? 0 : (nnz + kTile - 1) / kTile;
  P->ntiles = ntiles;
  if (ntiles == 0)
    return LA_OK;
  const int *ai = A->h_ai.data();
  std::vector<int> trow(ntiles + 1);
  for (int t = 0; t <= ntiles; t++) {
    const long k = std::min<long>((long)t * kTile, nnz);
    trow[t] = int(std::upper_bound(ai, ai + n + 1, (int)(k + base)) - ai) - 1;
  }
  LA_TRY(P->tile_row.upload(trow.data(), sizeof(int) * trow.size()));
  // merge groups: tiles [f, e) share head row trow[f]
  std::vector<int> gend(ntiles, -1);
  for (int f = 0; f < ntiles;) {
    int e = f + 1;
    while (e < ntiles && trow[e] == trow[f])
      e++;
    gend[f] = e;
    f = e;
  }
  LA_TRY(P->group_end.upload(gend.data(), sizeof(int) * gend.size()));
  P->h_tile_row = trow;
  P->h_group_end = gend;
  int longest = 0;
  for (int r = 0; r < n; r++)
    longest = std::max(longest, ai[r + 1] - ai[r]);
  P->long_rows = longest > kLongRow;
  P->vec_tiles = longest <= kVecRow;
  LA_TRY(P->part.alloc(sizeof(double) * 2 * ntiles));
  LA_CUDA_TRY(cudaMemset(P->part.p, 0, P->part.bytes));
  // the row-slot form: large matrices whose rows all hold at most kEllRow
  // entries and whose slots pad them by at most a quarter (measured on the
  // 128^3 Laplacian, FP64: 41.0 / 30.9 us with L2 flushed / back to back
  // against 52.3 / 45.3 us for the tile pass; 192^3 anisotropic: 120.9 /
  // 110.7 against 150.6 / 145.6 us).  LA_SPMV_ELL=0/1: testing / tuning
  // override (1 also below the size threshold)
  bool ell = n >= kEllMinRows && longest > 0 && longest <= kEllRow &&
             (long long)longest * n * 4 <= 5LL * nnz;
  if (const char *e = std::getenv("LA_SPMV_ELL"))
    ell = std::atoi(e) != 0 && longest <= kEllRow && longest > 0;
  if (ell) {
    const size_t cells = (size_t)longest * n;
    LA_TRY(P->ell_j.alloc(sizeof(int) * cells));
    const int g = std::max(1, std::min((n + kThreads - 1) / kThreads, 8 * sm_count()));
    if (A->dtype == LA_F64) {
      LA_TRY(P->ell_v.alloc(sizeof(double) * cells));
      ell_build_kernel<double><<<g, kThreads>>>(n, longest, base, A->ai.as<int>(),
                                                A->aj.as<int>(), A->av.as<double>(),
                                                P->ell_j.as<int>(), P->ell_v.as<double>());
    }
    if (const float *v32 = static_cast<const float *>(A->values(LA_F32))) {
      LA_TRY(P->ell_v32.alloc(sizeof(float) * cells));
      ell_build_kernel<float><<<g, kThreads>>>(n, longest, base, A->ai.as<int>(),
                                               A->aj.as<int>(), v32,
                                               A->dtype == LA_F64 ? nullptr : P->ell_j.as<int>(),
                                               P->ell_v32.as<float>());
    }
    LA_CUDA_TRY(cudaGetLastError());
    P->ell_k = longest;
  }
  return LA_OK;
}

int spmv_tile_nnz() { return kTile; }

// la_spmv_host, FP64: x in, the tiles in up to 8 chunks on one stream, and
// after each chunk the rows it finished -- those below the next chunk's first
// tile row; that row may still get partials -- copied out on a second stream,
// so the copy of y overlaps the rest of the computation.  The same tiles,
// partials and merge order as one launch: bit-identical to la_spmv.
la_status spmv_host_chunked(la_spmv_plan_t P, double alpha, const double *x, double beta,
                            double *y) {
  const la_csr_t A = P->A;
  const int n = A->n;
  if (!P->hx.p) {
    LA_TRY(P->hx.alloc(sizeof(double) * std::max(A->ncols, 1)));
    LA_TRY(P->hy.alloc(sizeof(double) * std::max(n, 1)));
    // blocking streams: ordered after work on the legacy default stream, as
    // the synchronous copies of this call always were
    LA_CUDA_TRY(cudaStreamCreate(&P->hst));
    LA_CUDA_TRY(cudaStreamCreate(&P->hcp));
    for (cudaEvent_t &e : P->hev)
      LA_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  double *hx = P->hx.as<double>(), *hy = P->hy.as<double>();
  LA_CUDA_TRY(cudaMemcpyAsync(hx, x, sizeof(double) * A->ncols, cudaMemcpyHostToDevice, P->hst));
  if (beta != 0.0)
    LA_CUDA_TRY(cudaMemcpyAsync(hy, y, sizeof(double) * n, cudaMemcpyHostToDevice, P->hst));
  // chunks of at least 64 tiles (64K nonzeros): below that the launches and
  // copies of a chunk cost more than the overlap returns
  const int nt = P->ntiles, chunks = std::min(8, nt / 64);
  if (chunks <= 1 || A->dtype != LA_F64 || P->ell_k) {
    LA_TRY(spmv_launch(P, alpha, hx, beta, hy, hy, LA_F64, P->hst));
    LA_CUDA_TRY(cudaMemcpyAsync(y, hy, sizeof(double) * n, cudaMemcpyDeviceToHost, P->hst));
    LA_CUDA_TRY(cudaStreamSynchronize(P->hst));
    return LA_OK;
  }
  const double *av = A->av.as<double>();
  for (int c = 0; c < chunks; c++) {
    const int t0 = (int)((long long)nt * c / chunks), t1 = (int)((long long)nt * (c + 1) / chunks);
    la_status s = P->kind == LA_SPMV_ALBUS
                      ? launch_form<kAlbus>(P, av, alpha, (const double *)hx, beta, hy,
                                            (const double *)hy, P->hst, XParts<double>{}, t0, t1)
                      : launch_form<kSegSum>(P, av, alpha, (const double *)hx, beta, hy,
                                             (const double *)hy, P->hst, XParts<double>{}, t0,
                                             t1);
    LA_TRY(s);
    const int r0 = c == 0 ? 0 : P->h_tile_row[t0], r1 = c == chunks - 1 ? n : P->h_tile_row[t1];
    LA_CUDA_TRY(cudaEventRecord(P->hev[c], P->hst));
    LA_CUDA_TRY(cudaStreamWaitEvent(P->hcp, P->hev[c], 0));
    if (r1 > r0)
      LA_CUDA_TRY(cudaMemcpyAsync(y + r0, hy + r0, sizeof(double) * (r1 - r0),
                                  cudaMemcpyDeviceToHost, P->hcp));
  }
  LA_CUDA_TRY(cudaStreamSynchronize(P->hcp));
  LA_CUDA_TRY(cudaStreamSynchronize(P->hst));
  return LA_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free SpMV (la_spmv_noalloc).  The per-call scratch of the tile
// pass -- the row holding each tile's first nonzero and the head / tail
// partial sums -- lives in this file-scope device array instead of plan
// memory, so a call allocates nothing.  Capacity: kNoAllocMaxTiles tiles,
// i.e. nnz <= kNoAllocMaxTiles * kTile = 33,554,432.  Every GPU that loads
// the library holds the array (655,616 bytes) until the process exits.  All
// calls share it: a call rewrites every entry it reads (nothing has to start
// at zero), and calls whose kernels overlap on the GPU race on it.
namespace {
constexpr int kNoAllocMaxTiles = 32768;
constexpr size_t kNoAllocPartBytes = sizeof(double) * 2 * kNoAllocMaxTiles;
constexpr size_t kNoAllocBytes =
    (kNoAllocPartBytes + sizeof(int) * (kNoAllocMaxTiles + 1) + 255) / 256 * 256;
static __device__ __align__(256) unsigned char g_spmv_scratch[kNoAllocBytes];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void *g_noalloc_addr[kMaxDevices] = {};

// Device address of g_spmv_scratch on the current device.  In host code the
// array's name is only a host-side stand-in, so the address is looked up
// once per device (the first call on that device) with that device current.
la_status noalloc_scratch(void **out) {
  int dev = 0;
  LA_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("device ordinal %d out of range", dev);
    return LA_ERR_INVALID_ARG;
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void *p = nullptr;
    LA_CUDA_TRY(cudaGetSymbolAddress(&p, g_spmv_scratch));
    g_noalloc_addr[dev] = p;
  }
  *out = g_noalloc_addr[dev];
  return LA_OK;
}

// tile_row[t] = upper_bound(ai, min(t * kTile, nnz) + base) - 1, t <= ntiles.
// The arrays come straight from the caller, so nothing on the host has
// checked that ai[0] == base and ai[n] - base == nnz.  The rows are clamped
// so that a violation can never send a write outside y[0, n): a tile's first
// row to [0, n - 1] (the merge writes y at it), the end row to [0, n].  With
// nnz > ai[n] - base the surplus tiles then hold empty segments of row n - 1
// (their aj / av reads stay below the nnz the caller declared).
__global__ void noalloc_tile_row_kernel(const int n, const int nnz, const int base,
                                        const int *__restrict__ ai, const int ntiles,
                                        int *tile_row) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t > ntiles)
    return;
  const int k = min(t * kTile, nnz) + base;
  int lo = 0, hi = n + 1;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(ai + mid) > k)
      hi = mid;
    else
      lo = mid + 1;
  }
  tile_row[t] = max(0, min(lo - 1, t < ntiles ? n - 1 : n));
}

template <int FORM>
la_status noalloc_launch(int n, int nnz, int base, const int *ai, const int *aj,
                         const double *av, double alpha, const double *x, double beta,
                         double *y, cudaStream_t st) {
  if (n == 0)
    return LA_OK;
  if (nnz == 0) {
    spmv_empty_kernel<double, double><<<std::min((n + 255) / 256, 4096), 256, 0, st>>>(
        n, y, y, beta);
    LA_CUDA_TRY(cudaGetLastError());
    return LA_OK;
  }
  void *scratch = nullptr;
  LA_TRY(noalloc_scratch(&scratch));
  double *part = static_cast<double *>(scratch);
  int *tile_row = reinterpret_cast<int *>(static_cast<unsigned char *>(scratch) +
                                          kNoAllocPartBytes);
  const int ntiles = (nnz + kTile - 1) / kTile;
  noalloc_tile_row_kernel<<<(ntiles + 1 + 255) / 256, 256, 0, st>>>(n, nnz, base, ai,
                                                                      ntiles, tile_row);
  LA_CUDA_TRY(cudaGetLastError());
  spmv_tile_kernel<FORM, double, double, double><<<ntiles, kThreads, 0, st>>>(
      n, nnz, base, ai, aj, av, x, y, y, alpha, beta, tile_row, part);
  LA_CUDA_TRY(cudaGetLastError());
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((ntiles + 255) / 256);
  cfg.blockDim = dim3(256);
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  const double *yin = y, *pt = part;
  const int *tr = tile_row, *ge = nullptr;
  const int f0 = 0, t0 = 0, t1 = ntiles;
  LA_CUDA_TRY(cudaLaunchKernelEx(&cfg, spmv_merge_kernel<FORM, double, double>, ntiles, y,
                                 yin, beta, tr, pt, ge, f0, t0, t1));
  return LA_OK;
}
} // namespace

la_status spmv_noalloc(la_spmv_kind kind, int n, int nnz, int base, const int *ai,
                       const int *aj, const double *av, double alpha, const double *x,
                       double beta, double *y, cudaStream_t st) {
  if (nnz > kNoAllocMaxTiles * kTile) {
    set_error("la_spmv_noalloc: nnz %d exceeds the allocation-free limit of %d "
              "(use la_spmv with a plan)", nnz, kNoAllocMaxTiles * kTile);
    return LA_ERR_INVALID_ARG;
  }
  if (kind == LA_SPMV_ALBUS)
    return noalloc_launch<kAlbus>(n, nnz, base, ai, aj, av, alpha, x, beta, y, st);
  return noalloc_launch<kSegSum>(n, nnz, base, ai, aj, av, alpha, x, beta, y, st);
}

} // namespace la
