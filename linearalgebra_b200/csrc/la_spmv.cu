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
// B200 design.  A "tile" is 2048 consecutive nonzeros (256 threads x 8);
// the plan stores the row that holds each tile's first nonzero (the
// reference's ALBUS preprocess, spmv.hpp:210-217).  Each thread streams its
// 8 values and 8 column indices with 128-bit non-allocating loads, gathers
// x through the read-only path (L1/L2; x of every configuration here fits
// in the 126 MB L2), and walks its rows sequentially.  Row partials that
// cross thread boundaries are joined by a CTA segmented scan (warp shuffles
// + shared memory) -- the GPU analogue of the reference's carry scan.  A row
// that crosses a tile boundary is finalised by whichever of its tiles
// arrives last at a per-row counter (atomicAdd after a device fence); that
// tile sums the partials in tile order, writes y and resets the counter.
// There is no spin-wait anywhere and the result is deterministic.
//
// Roofline: HBM-bound.  Algorithmic bytes per call
//   nnz*(sizeof(V) + 4) + (n+1)*4 + n*sizeof(X) [x] + n*sizeof(X) [y]
//   (+ n*sizeof(X) when beta != 0).

#include "la_device.cuh"
#include "la_internal.h"

#include <algorithm>
#include <cstring>

namespace la {
namespace {

constexpr int kThreads = 256;
constexpr int kNpt = 8;                  // nonzeros per thread
constexpr int kTile = kThreads * kNpt;   // nonzeros per tile

template <typename V> struct Vals8;
template <> struct Vals8<double> {
  static __device__ __forceinline__ void load(const double *p, double (&v)[kNpt]) {
    const double2 *q = reinterpret_cast<const double2 *>(p);
#pragma unroll
    for (int i = 0; i < kNpt / 2; i++) {
      const double2 t = dev::ld_stream(q + i);
      v[2 * i] = t.x;
      v[2 * i + 1] = t.y;
    }
  }
};
template <> struct Vals8<float> {
  static __device__ __forceinline__ void load(const float *p, float (&v)[kNpt]) {
    const float4 *q = reinterpret_cast<const float4 *>(p);
#pragma unroll
    for (int i = 0; i < kNpt / 4; i++) {
      const float4 t = dev::ld_stream(q + i);
      v[4 * i] = t.x;
      v[4 * i + 1] = t.y;
      v[4 * i + 2] = t.z;
      v[4 * i + 3] = t.w;
    }
  }
};
__device__ __forceinline__ void load_cols8(const int *p, int (&c)[kNpt]) {
  const int4 *q = reinterpret_cast<const int4 *>(p);
#pragma unroll
  for (int i = 0; i < kNpt / 4; i++) {
    const int4 t = dev::ld_stream(q + i);
    c[4 * i] = t.x;
    c[4 * i + 1] = t.y;
    c[4 * i + 2] = t.z;
    c[4 * i + 3] = t.w;
  }
}

enum Form { kSegSum = 0, kAlbus = 1 };

// Last row r in [lo, hi] with ai[r] - base <= k: the row holding nonzero k.
__device__ __forceinline__ int row_of(const int *__restrict__ ai, int base,
                                      int lo, int hi, int k) {
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(ai + mid) - base <= k)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

template <int FORM, typename ACC> struct RowOut {
  ACC alpha, beta;
  // A whole row finished inside one tile.
  template <typename X>
  __device__ __forceinline__ void write(X *y, const X *yin, int r, ACC sum) const {
    const ACC b = beta == ACC(0) ? ACC(0) : beta * ACC(yin[r]);
    y[r] = X(FORM == kAlbus ? alpha * sum + b : sum + b);
  }
  // A partial row handed to the cross-tile merge.
  __device__ __forceinline__ ACC partial(ACC sum) const {
    return FORM == kAlbus ? alpha * sum : sum;
  }
};

// One tile per CTA.  y = alpha*A*x + beta*yin (yin may equal y).
template <int FORM, typename V, typename X, typename ACC>
__global__ void __launch_bounds__(kThreads)
    spmv_tile_kernel(const int n, const int nnz, const int base,
                     const int *__restrict__ ai, const int *__restrict__ aj,
                     const V *__restrict__ av, const X *__restrict__ x, X *y,
                     const X *yin, const ACC alpha, const ACC beta,
                     const int *__restrict__ tile_row,
                     const int *__restrict__ head_slot,
                     const int *__restrict__ slot_cnt, ACC *part,
                     unsigned *arrive, const int ntiles) {
  __shared__ dev::SegPair<ACC> warp_tot[kThreads / 32];
  const RowOut<FORM, ACC> out{alpha, beta};
  const int t = blockIdx.x;
  const int s = t * kTile;
  const int e = min(s + kTile, nnz);
  const int R0 = __ldg(tile_row + t), R1 = __ldg(tile_row + t + 1);
  const int k0 = s + threadIdx.x * kNpt;
  const int cnt = max(0, min(kNpt, e - k0));

  if (t == 0) // leading empty rows (ai[r + 1] == ai[0]) precede tile 0
    for (int r = threadIdx.x; r < R0; r += kThreads)
      out.write(y, yin, r, ACC(0));

  ACC p[kNpt];
  if (cnt == kNpt) {
    V v[kNpt];
    int c[kNpt];
    Vals8<V>::load(av + k0, v);
    load_cols8(aj + k0, c);
#pragma unroll
    for (int q = 0; q < kNpt; q++) {
      const ACC xv = ACC(__ldg(x + c[q] - base));
      p[q] = FORM == kSegSum ? (alpha * ACC(v[q])) * xv : ACC(v[q]) * xv;
    }
  } else {
#pragma unroll
    for (int q = 0; q < kNpt; q++) {
      p[q] = ACC(0);
      if (q < cnt) {
        const ACC xv = ACC(__ldg(x + __ldg(aj + k0 + q) - base));
        const ACC vv = ACC(__ldg(av + k0 + q));
        p[q] = FORM == kSegSum ? (alpha * vv) * xv : vv * xv;
      }
    }
  }

  // Sequential walk over this thread's nonzeros.  The first row that ends
  // here may have started in an earlier thread: keep it as `lead` until the
  // CTA scan supplies its carry.  Later rows are whole: write them.
  dev::SegPair<ACC> me{0, ACC(0)};
  ACC lead = ACC(0);
  int lead_row = -1;
  if (cnt > 0) {
    int r = threadIdx.x == 0 ? R0 : row_of(ai, base, R0, R1, k0);
    int next_end = __ldg(ai + r + 1) - base;
    ACC acc = ACC(0);
#pragma unroll
    for (int q = 0; q < kNpt; q++) {
      if (q < cnt) {
        acc += p[q];
        const int kend = k0 + q + 1;
        while (next_end == kend) {
          if (!me.f) {
            me.f = 1;
            lead = acc;
            lead_row = r;
          } else {
            out.write(y, yin, r, acc);
          }
          acc = ACC(0);
          if (++r >= n)
            break;
          next_end = __ldg(ai + r + 1) - base;
        }
      }
    }
    me.v = acc;
  }

  // CTA-wide exclusive segmented scan of (row ended?, trailing partial).
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const dev::SegPair<ACC> inc = dev::warp_seg_scan_incl(me);
  if (lane == 31)
    warp_tot[warp] = inc;
  dev::SegPair<ACC> ex;
  ex.f = __shfl_up_sync(0xffffffffu, inc.f, 1);
  ex.v = __shfl_up_sync(0xffffffffu, inc.v, 1);
  if (lane == 0) {
    ex.f = 0;
    ex.v = ACC(0);
  }
  __syncthreads();
  dev::SegPair<ACC> carry{0, ACC(0)};
  for (int w = 0; w < warp; w++) {
    const dev::SegPair<ACC> b = warp_tot[w];
    carry.v = b.f ? b.v : carry.v + b.v;
    carry.f |= b.f;
  }
  carry.v = ex.f ? ex.v : carry.v + ex.v;
  carry.f |= ex.f;

  if (me.f) {
    const ACC val = lead + carry.v;
    if (!carry.f) { // first row end of the tile: the tile's head row R0
      part[2 * t] = out.partial(val);
      __threadfence();
    } else {
      out.write(y, yin, lead_row, val);
    }
  }

  if (threadIdx.x == 0) {
    dev::SegPair<ACC> tot{0, ACC(0)};
    for (int w = 0; w < kThreads / 32; w++) {
      const dev::SegPair<ACC> b = warp_tot[w];
      tot.v = b.f ? b.v : tot.v + b.v;
      tot.f |= b.f;
    }
    if (tot.f) {
      if (R1 < n)
        part[2 * t + 1] = out.partial(tot.v); // partial first part of R1
    } else {
      part[2 * t] = out.partial(tot.v); // the whole tile lies inside R0
    }
  }
  __syncthreads(); // the head partial written by another thread is fenced
  if (threadIdx.x != 0)
    return;
  __threadfence();

  // Arrive at the merge slot of the head row and, if a row ends here, at the
  // slot of the tail row (tile t + 1 is the first tile holding it).  The
  // last contributor sums the partials in tile order and writes y.
  int slots[2] = {__ldg(head_slot + t), -1};
  if (R1 != R0 && R1 < n && t + 1 < ntiles)
    slots[1] = t + 1;
  for (int i = 0; i < 2; i++) {
    const int f = slots[i];
    if (f < 0)
      continue;
    const unsigned need = (unsigned)__ldg(slot_cnt + f);
    if (atomicAdd(arrive + f, 1u) + 1u != need)
      continue;
    __threadfence();
    arrive[f] = 0u;
    const int R = __ldg(tile_row + f);
    const ACC yb = beta == ACC(0) ? ACC(0) : beta * ACC(yin[R]);
    if (FORM == kAlbus) { // merge order of spmv.hpp:275-292
      ACC v = yb;
      if (f > 0)
        v += __ldcg(part + 2 * (f - 1) + 1);
      for (int u = f; u < ntiles && __ldg(tile_row + u) == R; u++)
        v += __ldcg(part + 2 * u);
      y[R] = X(v);
    } else { // carry chain of spmv.hpp:118-141, then + beta*x (:171)
      ACC c = f > 0 ? __ldcg(part + 2 * (f - 1) + 1) : ACC(0);
      for (int u = f; u < ntiles && __ldg(tile_row + u) == R; u++)
        c = __ldcg(part + 2 * u) + c;
      y[R] = X(c + yb);
    }
  }
}

// nnz == 0: every row is empty.
template <typename X, typename ACC>
__global__ void spmv_empty_kernel(int n, X *y, const X *yin, ACC beta) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n;
       r += gridDim.x * blockDim.x)
    y[r] = X(beta == ACC(0) ? ACC(0) : beta * ACC(yin[r]));
}

// dv[k] = alpha * g[row(k)] * x[col(k)] over the stored pattern.
__global__ void __launch_bounds__(kThreads)
    sddmm_kernel(const int n, const int nnz, const int base,
                 const int *__restrict__ ai, const int *__restrict__ aj,
                 const double *__restrict__ g, const double *__restrict__ x,
                 double *__restrict__ dv, const double alpha,
                 const int *__restrict__ tile_row) {
  const int t = blockIdx.x;
  const int s = t * kTile;
  const int e = min(s + kTile, nnz);
  const int k0 = s + threadIdx.x * kNpt;
  const int cnt = max(0, min(kNpt, e - k0));
  if (cnt == 0)
    return;
  int r = row_of(ai, base, __ldg(tile_row + t), __ldg(tile_row + t + 1), k0);
  int next_end = __ldg(ai + r + 1) - base;
  double out[kNpt];
#pragma unroll
  for (int q = 0; q < kNpt; q++) {
    out[q] = 0.0;
    if (q < cnt) {
      const int k = k0 + q;
      while (next_end <= k && r + 1 < n) {
        r++;
        next_end = __ldg(ai + r + 1) - base;
      }
      out[q] = alpha * __ldg(g + r) * __ldg(x + __ldg(aj + k) - base);
    }
  }
  if (cnt == kNpt) {
    double2 *d2 = reinterpret_cast<double2 *>(dv + k0);
#pragma unroll
    for (int i = 0; i < kNpt / 2; i++)
      d2[i] = make_double2(out[2 * i], out[2 * i + 1]);
  } else {
    for (int q = 0; q < cnt; q++)
      dv[k0 + q] = out[q];
  }
}

template <int FORM, typename V, typename X, typename ACC>
la_status launch_form(la_spmv_plan_t P, const V *av, ACC alpha, const X *x,
                      ACC beta, X *y, const X *yin, cudaStream_t st) {
  const la_csr_t A = P->A;
  if (A->n == 0)
    return LA_OK;
  if (A->nnz == 0) {
    spmv_empty_kernel<X, ACC><<<std::min((A->n + 255) / 256, 4096), 256, 0, st>>>(
        A->n, y, yin, beta);
  } else {
    spmv_tile_kernel<FORM, V, X, ACC><<<P->ntiles, kThreads, 0, st>>>(
        A->n, A->nnz, A->base, A->ai.as<int>(), A->aj.as<int>(), av, x, y, yin,
        alpha, beta, P->tile_row.as<int>(), P->head_slot.as<int>(),
        P->slot_cnt.as<int>(), P->part.as<ACC>(), P->arrive.as<unsigned>(),
        P->ntiles);
  }
  LA_CUDA_TRY(cudaGetLastError());
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
  if (P->kind == LA_SPMV_ALBUS)
    return launch_form<kAlbus>(P, av, fa, (const float *)x, fb, (float *)y,
                               (const float *)yin, st);
  return launch_form<kSegSum>(P, av, fa, (const float *)x, fb, (float *)y,
                              (const float *)yin, st);
}

la_status sddmm_launch(la_spmv_plan_t P, double alpha, const double *g,
                       const double *x, double *dv, cudaStream_t st) {
  const la_csr_t A = P->A;
  if (A->nnz == 0)
    return LA_OK;
  sddmm_kernel<<<P->ntiles, kThreads, 0, st>>>(
      A->n, A->nnz, A->base, A->ai.as<int>(), A->aj.as<int>(), g, x, dv, alpha,
      P->tile_row.as<int>());
  LA_CUDA_TRY(cudaGetLastError());
  return LA_OK;
}

// Plan: tile start rows (upper_bound on ai, as ALBUSSPMV::preprocess does,
// spmv.hpp:210-217), merge slots and per-slot contributor counts.
la_status spmv_plan_build(la_spmv_plan_t P) {
  const la_csr_t A = P->A;
  const int n = A->n, nnz = A->nnz, base = A->base;
  const int ntiles = nnz == 0 ? 0 : (nnz + kTile - 1) / kTile;
  P->ntiles = ntiles;
  if (ntiles == 0)
    return LA_OK;
  const int *ai = A->h_ai.data();
  std::vector<int> trow(ntiles + 1), hslot(ntiles), scnt(ntiles + 1, 0);
  for (int t = 0; t <= ntiles; t++) {
    const long k = std::min<long>((long)t * kTile, nnz);
    trow[t] = int(std::upper_bound(ai, ai + n + 1, (int)(k + base)) - ai) - 1;
  }
  for (int t = 0; t < ntiles; t++) {
    hslot[t] = (t > 0 && trow[t - 1] == trow[t]) ? hslot[t - 1] : t;
    scnt[hslot[t]]++;
  }
  for (int t = 1; t < ntiles; t++)
    if (hslot[t] == t)
      scnt[t]++; // the previous tile's tail partial
  LA_TRY(P->tile_row.upload(trow.data(), sizeof(int) * trow.size()));
  LA_TRY(P->head_slot.upload(hslot.data(), sizeof(int) * hslot.size()));
  LA_TRY(P->slot_cnt.upload(scnt.data(), sizeof(int) * scnt.size()));
  LA_TRY(P->part.alloc(sizeof(double) * 2 * ntiles));
  LA_TRY(P->arrive.alloc(sizeof(unsigned) * (ntiles + 1)));
  LA_CUDA_TRY(cudaMemset(P->arrive.p, 0, P->arrive.bytes));
  LA_CUDA_TRY(cudaMemset(P->part.p, 0, P->part.bytes));
  return LA_OK;
}

int spmv_tile_nnz() { return kTile; }

} // namespace la
