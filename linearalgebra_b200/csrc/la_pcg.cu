// la_pcg.cu -- IC(0)-preconditioned CG on one B200, FP64 and mixed.
//
// Reference: the reference's intended solve sequence (execs/linearSolve.cpp:
// 118-135): an IC(0) factor U of the SPD matrix (A ~= U^T U,
// incomplete_cholesky_k_2, mkl_wrapper/incomplete_cholesky.cpp:286-342),
// MKL's RCI PCG (mkl_wrapper/mkl_solver.cpp:150-251) with the preconditioner
// applied as trsv(U^T) then trsv(U) (incomplete_cholesky.cpp:21-29) and the
// user stopping test ||A x - b|| / ||b|| < rel_tol (mkl_solver.cpp:211-225).
// MKL is replaced by this file's loop over the library's own kernels: the
// nnz-balanced SpMV (la_spmv.cu), the persistent level-scheduled triangular
// solves (la_trsv.cu) and deterministic FP64 dot products below.
//
// Stopping: the recurrence residual is watched every iteration; once it is
// below rtol the true residual b - A x is formed in FP64 and the solve stops
// only if that is below rtol too (the reference's test, evaluated where it
// can change the outcome instead of after every iteration).
//
// Mixed mode: FP64 iterative refinement by reliable updates (pcg_mixed):
// the CG recurrence runs on FP32 vectors with FP32 matrix / factors, and the
// FP64 residual b - A x, FP64 update of x and FP64 dot products and norms
// recover the accuracy without restarting the Krylov space.

#include "la_device.cuh"
#include "la_internal.h"

#include <cmath>
#include <cstdlib>
#include <memory>
#include <utility>

namespace la {

la_status spmv_launch(la_spmv_plan_t P, double alpha, const void *x,
                      double beta, void *y, const void *yin, la_dtype vd,
                      cudaStream_t st);
la_status trsv_launch(la_trsv_plan_t P, const void *b, void *x,
                      cudaStream_t st);
la_status trsv_check(la_trsv_plan_t P, cudaStream_t st);
la_status trsv_build(la_trsv_plan_t P, const int *ai, const int *aj,
                     const double *av, const double *diag, const int *iperm = nullptr,
                     const int *prefix = nullptr, int nlevels = 0);
la_status spmv_plan_build(la_spmv_plan_t P);

namespace {

constexpr int kDotThreads = 512;

// Scalar slots in device memory.
enum { S_RZ = 0, S_PQ, S_RR, S_ALPHA, S_BETA, S_DOT, S_RZ0, S_COUNT };

// Deterministic FP64 dot with a fused finaliser: every block writes its
// partial sum, the last block to finish (atomic ticket after a fence) adds
// the partials in block order and applies `op`.
enum DotOp { OP_STORE = 0, OP_ALPHA = 1, OP_BETA = 2 };

// One block's share of a dot product, in the order every dot here uses:
// each thread's running sum s (its elements i = block * kDotThreads + tid +
// k * grid * kDotThreads, accumulated by fused multiply-adds in k order),
// a shuffle tree inside each warp, then the warps' sums in warp order.  The
// block total lands in thread 0's return value.
__device__ __forceinline__ double block_sum(double s, double *red) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1)
    s += __shfl_down_sync(0xffffffffu, s, d);
  if ((threadIdx.x & 31) == 0)
    red[threadIdx.x >> 5] = s;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < kDotThreads / 32; w++)
      t += red[w];
  return t;
}

// A thread's running sum over its elements i = block * kDotThreads + tid +
// k * stride, in k order; four elements are loaded before their four
// multiply-adds, so more loads are in flight and the order is unchanged.
template <typename XA, typename XB>
__device__ __forceinline__ double thread_dot(const int n, const XA *__restrict__ a,
                                             const XB *__restrict__ b) {
  const int stride = gridDim.x * kDotThreads;
  int i = blockIdx.x * kDotThreads + threadIdx.x;
  double s = 0.0;
  for (; i + 3 * stride < n; i += 4 * stride) {
    double u[4], v[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      u[k] = double(a[i + k * stride]);
      v[k] = double(b[i + k * stride]);
    }
#pragma unroll
    for (int k = 0; k < 4; k++)
      s = __fma_rn(u[k], v[k], s);
  }
  for (; i < n; i += stride)
    s = __fma_rn(double(a[i]), double(b[i]), s);
  return s;
}

// The block totals of `partials` (`count` of them) added in block order.
__device__ __forceinline__ double sum_partials(const double *partials, int count) {
  double t = 0.0;
  for (int k = 0; k < count; k++)
    t += __ldcg(partials + k);
  return t;
}

template <typename XA, typename XB>
__global__ void __launch_bounds__(kDotThreads)
    dot_kernel(const int n, const XA *__restrict__ a, const XB *__restrict__ b,
               double *partials, unsigned *ticket, double *scal, const int op) {
  __shared__ double red[kDotThreads / 32];
  __shared__ bool last;
  const double s = thread_dot(n, a, b);
  const double bt = block_sum(s, red);
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = bt;
    __threadfence();
    last = atomicAdd(ticket, 1u) + 1u == gridDim.x;
  }
  __syncthreads();
  if (!last || threadIdx.x != 0)
    return;
  __threadfence();
  const double t = sum_partials(partials, gridDim.x);
  *ticket = 0u;
  scal[S_DOT] = t;
  if (op == OP_ALPHA) { // alpha = (r, z) / (p, A p)
    scal[S_PQ] = t;
    scal[S_ALPHA] = scal[S_RZ] / t;
  } else if (op == OP_BETA) { // beta = (r, z)_new / (r, z)_old
    scal[S_BETA] = t / scal[S_RZ];
    scal[S_RZ0] = scal[S_RZ]; // kept so that a discarded step can be redone
    scal[S_RZ] = t;
  }
}

// x += alpha p; r -= alpha q (alpha from device memory).
template <typename X>
__global__ void xr_update_kernel(const int n, X *x, X *r, const X *p,
                                 const X *q, const double *scal) {
  const double al = scal[S_ALPHA];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x) {
    x[i] = X(__fma_rn(al, double(p[i]), double(x[i])));
    r[i] = X(__fma_rn(-al, double(q[i]), double(r[i])));
  }
}

// pn = z + beta p (out of place: the mixed loop may discard the result)
template <typename X>
__global__ void p_next_kernel(const int n, X *pn, const X *p, const X *z,
                              const double *scal) {
  const double be = scal[S_BETA];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x)
    pn[i] = X(__fma_rn(be, double(p[i]), double(z[i])));
}

// p = z + beta p
template <typename X>
__global__ void p_update_kernel(const int n, X *p, const X *z,
                                const double *scal) {
  const double be = scal[S_BETA];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x)
    p[i] = X(__fma_rn(be, double(p[i]), double(z[i])));
}

// ------------------------------------------------------ fused iteration
// One cooperative kernel carries the step after the SpMV (the role of the
// RCI loop's dot products and axpys there, mkl_solver.cpp:190-238):
//   pcg_update_kernel: alpha = (r, z) / (p, q); x += alpha p; r -= alpha q;
//                      ||r||^2 -- three launches of the unfused sequence.
// Its first dot product ends in a grid-wide barrier, after which every block
// adds the block totals itself, in block order, so no extra launch finishes
// it; the last one is finished by the last block, as in dot_kernel.  Grid,
// element assignment, per-thread order and reduction tree are dot_kernel's,
// and each update is the same single fused multiply-add as in
// xr_update_kernel: the iterates are bit-identical to the unfused sequence's.
// Launched cooperatively (all blocks resident); the barrier's wait is bounded
// by the global timer.  Measured on the 128^3 workload (us per iteration,
// events between launches): this kernel 54.0 against 56.3 for the three it
// replaces.  Two further fusions measured slower and are not used: the
// direction step as one cooperative kernel (beta and p = z + beta p after a
// grid barrier: 38.2 against 28.3 for dot_kernel + p_update_kernel), and the
// solves' sentinel fill folded into this kernel (the partitioned solves then
// took 470 / 475 instead of 454 / 454 -- their outputs are no longer hot in
// L2 when written amid this kernel's other traffic, where a memset right
// before each solve leaves them there).
// partials: 2 * gridDim.x doubles ((p, q) totals, then ||r||^2 totals).
template <typename X>
__global__ void __launch_bounds__(kDotThreads)
    pcg_update_kernel(const int n, X *x, X *r, const X *__restrict__ p,
                      const X *__restrict__ q, double *partials, unsigned *ticket,
                      double *scal, unsigned *bar) {
  __shared__ double red[kDotThreads / 32];
  __shared__ double alpha_s;
  __shared__ bool last;
  const int stride = gridDim.x * kDotThreads, i0 = blockIdx.x * kDotThreads + threadIdx.x;
  double s = thread_dot(n, p, q);
  const double bt = block_sum(s, red);
  if (threadIdx.x == 0)
    partials[blockIdx.x] = bt;
  dev::grid_barrier(bar);
  if (threadIdx.x == 0) {
    const double pq = sum_partials(partials, gridDim.x);
    const double al = scal[S_RZ] / pq; // alpha = (r, z) / (p, A p)
    alpha_s = al;
    if (blockIdx.x == 0) {
      scal[S_PQ] = pq;
      scal[S_ALPHA] = al;
    }
  }
  __syncthreads();
  const double al = alpha_s;
  s = 0.0;
  auto step = [&](int i, X pi, X qi, X xi, X ri) {
    x[i] = X(__fma_rn(al, double(pi), double(xi)));
    const X rn = X(__fma_rn(-al, double(qi), double(ri)));
    r[i] = rn;
    s = __fma_rn(double(rn), double(rn), s);
  };
  int i = i0;
  for (; i + 3 * stride < n; i += 4 * stride) { // loads first, then the k-order steps
    X pv[4], qv[4], xv[4], rv[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const int j = i + k * stride;
      pv[k] = p[j];
      qv[k] = q[j];
      xv[k] = x[j];
      rv[k] = r[j];
    }
#pragma unroll
    for (int k = 0; k < 4; k++)
      step(i + k * stride, pv[k], qv[k], xv[k], rv[k]);
  }
  for (; i < n; i += stride)
    step(i, p[i], q[i], x[i], r[i]);
  const double bt2 = block_sum(s, red);
  if (threadIdx.x == 0) {
    partials[gridDim.x + blockIdx.x] = bt2;
    __threadfence();
    last = atomicAdd(ticket, 1u) + 1u == gridDim.x;
  }
  __syncthreads();
  if (!last || threadIdx.x != 0)
    return;
  __threadfence();
  scal[S_DOT] = sum_partials(partials + gridDim.x, gridDim.x);
  *ticket = 0u;
}

// out = X(scale * in)
template <typename XO, typename XI>
__global__ void scale_copy_kernel(const int n, XO *out, const XI *in,
                                  const double scale) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x)
    out[i] = XO(scale * double(in[i]));
}

// x += scale * d
__global__ void refine_kernel(const int n, double *x, const float *d,
                              const double scale) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x)
    x[i] += scale * double(d[i]);
}

__global__ void zero_kernel(const int n, double *x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x)
    x[i] = 0.0;
}

} // namespace
} // namespace la



namespace la {
namespace {

int vec_grid(int n) { return std::max(1, std::min((n + 255) / 256, 8 * sm_count())); }

template <typename XA, typename XB>
la_status dot(la_pcg_t S, const XA *a, const XB *b, int op, cudaStream_t st) {
  dot_kernel<XA, XB><<<S->dot_blocks, kDotThreads, 0, st>>>(
      S->n, a, b, S->partials.as<double>(), S->ticket.as<unsigned>(),
      S->scal.as<double>(), op);
  LA_CUDA_TRY(cudaGetLastError());
  return LA_OK;
}

template <typename X>
la_status fused_update(la_pcg_t S, X *x, X *r, const X *p, const X *q, cudaStream_t st) {
  int n = S->n;
  double *partials = S->partials.as<double>(), *scal = S->scal.as<double>();
  unsigned *ticket = S->ticket.as<unsigned>(), *bar = S->bar.as<unsigned>();
  void *args[] = {&n, &x, &r, &p, &q, &partials, &ticket, &scal, &bar};
  LA_CUDA_TRY(cudaLaunchCooperativeKernel((const void *)pcg_update_kernel<X>,
                                          dim3(S->dot_blocks), dim3(kDotThreads), args, 0, st));
  return LA_OK;
}

// Reads (and clears) the fused kernels' barrier error word; synchronises st.
la_status barrier_check(la_pcg_t S, cudaStream_t st) {
  if (!S->fused)
    return LA_OK;
  unsigned h = 0;
  LA_CUDA_TRY(cudaMemcpyAsync(&h, S->bar.as<unsigned>() + 2, sizeof(unsigned),
                              cudaMemcpyDeviceToHost, st));
  LA_CUDA_TRY(cudaStreamSynchronize(st));
  if (h) {
    LA_CUDA_TRY(cudaMemsetAsync(S->bar.p, 0, S->bar.bytes, st));
    set_error("PCG: a grid-wide barrier wait exceeded its 1 s bound");
    return LA_ERR_TIMEOUT;
  }
  return LA_OK;
}

la_status read_scalar(la_pcg_t S, int slot, double *v, cudaStream_t st) {
  LA_CUDA_TRY(cudaMemcpyAsync(v, S->scal.as<double>() + slot, sizeof(double),
                              cudaMemcpyDeviceToHost, st));
  LA_CUDA_TRY(cudaStreamSynchronize(st));
  return LA_OK;
}

// True relative residual ||b - A x|| / bnorm in FP64 (uses t).
la_status true_residual(la_pcg_t S, const double *b, const double *x,
                        double bnorm, double *rel, cudaStream_t st) {
  LA_TRY(spmv_launch(S->Ap, -1.0, x, 1.0, S->t.p, b, LA_F64, st));
  LA_TRY(dot(S, S->t.as<double>(), S->t.as<double>(), OP_STORE, st));
  double tt;
  LA_TRY(read_scalar(S, S_DOT, &tt, st));
  *rel = std::sqrt(tt) / bnorm;
  return LA_OK;
}

// One preconditioned CG run on A y = rhs from y = 0 with vectors of type X.
// Stops when ||r|| <= tol * ||rhs|| (recurrence residual), or, when
// `b_true` is given (FP64 mode), when additionally the true residual of y
// against b_true is below tol.  Returns the iteration count in *iters.
template <typename X>
la_status pcg_run(la_pcg_t S, const X *rhs, X *y, X *r, X *z, X *p, X *q,
                  X *t, la_dtype vd, double tol, int maxit, const double *b_true,
                  double bnorm_true, int *iters, double *rel_out,
                  cudaStream_t st) {
  const int n = S->n, g = vec_grid(n);
  *iters = 0;
  LA_CUDA_TRY(cudaMemsetAsync(y, 0, sizeof(X) * n, st));
  LA_CUDA_TRY(cudaMemcpyAsync(r, rhs, sizeof(X) * n, cudaMemcpyDeviceToDevice, st));
  LA_TRY(dot(S, r, r, OP_STORE, st));
  double rr0;
  LA_TRY(read_scalar(S, S_DOT, &rr0, st));
  const double r0 = std::sqrt(rr0);
  if (r0 == 0.0) {
    *rel_out = 0.0;
    return LA_OK;
  }
  LA_TRY(trsv_launch(S->L, r, t, st));
  LA_TRY(trsv_launch(S->U, t, z, st));
  LA_CUDA_TRY(cudaMemcpyAsync(p, z, sizeof(X) * n, cudaMemcpyDeviceToDevice, st));
  LA_TRY(dot(S, r, z, OP_STORE, st));
  LA_CUDA_TRY(cudaMemcpyAsync(S->scal.as<double>() + S_RZ,
                              S->scal.as<double>() + S_DOT, sizeof(double),
                              cudaMemcpyDeviceToDevice, st));
  for (int it = 1; it <= maxit; it++) {
    LA_TRY(spmv_launch(S->Ap, 1.0, p, 0.0, q, q, vd, st));
    if (S->fused) {
      LA_TRY(fused_update<X>(S, y, r, p, q, st));
    } else {
      LA_TRY(dot(S, p, q, OP_ALPHA, st));
      xr_update_kernel<X><<<g, 256, 0, st>>>(n, y, r, p, q, S->scal.as<double>());
      LA_TRY(dot(S, r, r, OP_STORE, st));
    }
    // ||r||^2 travels to the host while the next iteration's preconditioner
    // and direction update are already queued behind it, so the GPU does
    // not idle through the host's check.  They write only t, z, p and the
    // rz scalar: when this iteration is the last, y and r are untouched.
    LA_CUDA_TRY(cudaMemcpyAsync(S->h_rr, S->scal.as<double>() + S_DOT, sizeof(double),
                                cudaMemcpyDeviceToHost, st));
    LA_CUDA_TRY(cudaEventRecord(S->ev_rr, st));
    LA_TRY(trsv_launch(S->L, r, t, st));
    LA_TRY(trsv_launch(S->U, t, z, st));
    LA_TRY(dot(S, r, z, OP_BETA, st));
    p_update_kernel<X><<<g, 256, 0, st>>>(n, p, z, S->scal.as<double>());
    LA_CUDA_TRY(cudaEventSynchronize(S->ev_rr));
    const double rr = *S->h_rr;
    *iters = it;
    const double rel = std::sqrt(rr) / r0;
    *rel_out = rel;
    if (!std::isfinite(rel)) {
      // a solve that gave up on a wait leaves sentinel NaNs behind: report
      // (and clear) the timeout rather than a breakdown it caused
      LA_TRY(trsv_check(S->L, st));
      LA_TRY(trsv_check(S->U, st));
      set_error("PCG breakdown: non-finite residual at iteration %d", it);
      return LA_ERR_BREAKDOWN;
    }
    if (rel < tol) {
      if (!b_true)
        return LA_OK;
      double trel;
      LA_TRY(true_residual(S, b_true, (const double *)y, bnorm_true, &trel, st));
      *rel_out = trel;
      if (trel < tol)
        return LA_OK;
    }
  }
  LA_TRY(trsv_check(S->L, st));
  LA_TRY(trsv_check(S->U, st));
  return LA_ERR_NOT_CONVERGED;
}

// Mixed precision with reliable updates (FP64 iterative refinement that
// keeps the Krylov space): the CG recurrence runs on FP32 vectors with the
// FP32 matrix and FP32 IC(0) factors (FP32 SpMV and triangular solves, FP32
// accumulation in those kernels), its dot products and scalars in FP64.  The
// FP32 iterate is a correction d accumulated since the last update; whenever
// the FP32 residual has fallen by a factor delta since then (or below rtol),
// x += d in FP64, the residual is recomputed as r = b - A x with the FP64
// matrix, and the FP32 residual is replaced by it -- without restarting the
// search direction, so the iteration count stays close to the FP64 solver's.
// The solve stops when that FP64 residual satisfies ||r|| / ||b|| < rtol.
// delta (S->reliable_delta) is 0.1 unless LA_PCG_RELIABLE_DELTA, a
// tuning override read when the solver is created, says otherwise.

la_status pcg_mixed(la_pcg_t S, const double *b, double *x, double bn, double rtol,
                    int maxit, la_pcg_info *loc, cudaStream_t st) {
  const int n = S->n, g = vec_grid(n);
  float *r32 = S->r32.as<float>(), *z32 = S->z32.as<float>(), *p32 = S->p32.as<float>(),
        *q32 = S->q32.as<float>(), *t32 = S->t32.as<float>(), *d32 = S->d32.as<float>(),
        *pn32 = S->p32b.as<float>();
  double *r64 = S->r.as<double>();
  zero_kernel<<<g, 256, 0, st>>>(n, x);
  LA_CUDA_TRY(cudaMemsetAsync(d32, 0, sizeof(float) * n, st));
  scale_copy_kernel<float, double><<<g, 256, 0, st>>>(n, r32, b, 1.0);
  LA_TRY(trsv_launch(S->L, r32, t32, st));
  LA_TRY(trsv_launch(S->U, t32, z32, st));
  LA_CUDA_TRY(cudaMemcpyAsync(p32, z32, sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
  LA_TRY(dot(S, r32, z32, OP_STORE, st));
  LA_CUDA_TRY(cudaMemcpyAsync(S->scal.as<double>() + S_RZ, S->scal.as<double>() + S_DOT,
                              sizeof(double), cudaMemcpyDeviceToDevice, st));
  double rmax = bn, rel = 1.0, rn_prev = bn;
  int updates = 0, it;
  for (it = 1; it <= maxit; it++) {
    LA_TRY(spmv_launch(S->Ap, 1.0, p32, 0.0, q32, q32, LA_F32, st));
    if (S->fused) {
      LA_TRY(fused_update<float>(S, d32, r32, p32, q32, st));
    } else {
      LA_TRY(dot(S, p32, q32, OP_ALPHA, st));
      xr_update_kernel<float><<<g, 256, 0, st>>>(n, d32, r32, p32, q32, S->scal.as<double>());
      LA_TRY(dot(S, r32, r32, OP_STORE, st));
    }
    // As in pcg_run: ||r||^2 travels to the host while the next step's
    // preconditioner and direction are queued -- when the last residual was
    // well above the reliable-update threshold, so that no update is likely
    // now (one iteration in about twenty has one, and a discarded step costs
    // two triangular solves).  The queued step writes t, z, the next
    // direction pn and the rz / beta scalars; if an update is due after all,
    // rz is restored and the step is redone on the new residual.
    LA_CUDA_TRY(cudaMemcpyAsync(S->h_rr, S->scal.as<double>() + S_DOT, sizeof(double),
                                cudaMemcpyDeviceToHost, st));
    LA_CUDA_TRY(cudaEventRecord(S->ev_rr, st));
    const bool ahead = rn_prev > S->ahead_margin * S->reliable_delta * rmax &&
                       rn_prev > 2.0 * rtol * bn;
    auto precondition = [&]() -> la_status {
      LA_TRY(trsv_launch(S->L, r32, t32, st));
      LA_TRY(trsv_launch(S->U, t32, z32, st));
      LA_TRY(dot(S, r32, z32, OP_BETA, st));
      p_next_kernel<float><<<g, 256, 0, st>>>(n, pn32, p32, z32, S->scal.as<double>());
      return LA_OK;
    };
    if (ahead)
      LA_TRY(precondition());
    LA_CUDA_TRY(cudaEventSynchronize(S->ev_rr));
    const double rr = *S->h_rr;
    const double rn = std::sqrt(rr);
    rn_prev = rn;
    bool updated = false;
    if (!std::isfinite(rn)) {
      loc->iterations = it;
      LA_TRY(trsv_check(S->L, st)); // a timed-out solve, not a breakdown
      LA_TRY(trsv_check(S->U, st));
      set_error("mixed PCG breakdown: non-finite residual at iteration %d", it);
      return LA_ERR_BREAKDOWN;
    }
    if (rn < S->reliable_delta * rmax || rn / bn < rtol) {
      refine_kernel<<<g, 256, 0, st>>>(n, x, d32, 1.0);
      LA_CUDA_TRY(cudaMemsetAsync(d32, 0, sizeof(float) * n, st));
      LA_TRY(spmv_launch(S->Ap, -1.0, x, 1.0, r64, b, LA_F64, st));
      LA_TRY(dot(S, r64, r64, OP_STORE, st));
      double rr64;
      LA_TRY(read_scalar(S, S_DOT, &rr64, st));
      rmax = std::sqrt(rr64);
      rel = rmax / bn;
      updates++;
      if (rel < rtol)
        break;
      scale_copy_kernel<float, double><<<g, 256, 0, st>>>(n, r32, r64, 1.0);
      updated = true;
    }
    if (ahead && updated) // the queued step used the old residual: redo it
      LA_CUDA_TRY(cudaMemcpyAsync(S->scal.as<double>() + S_RZ, S->scal.as<double>() + S_RZ0,
                                  sizeof(double), cudaMemcpyDeviceToDevice, st));
    if (!ahead || updated)
      LA_TRY(precondition());
    std::swap(p32, pn32);
  }
  loc->iterations = std::min(it, maxit);
  loc->outer_iterations = updates;
  loc->rel_residual = rel;
  if (rel >= rtol) {
    // final FP64 residual of the last iterate
    refine_kernel<<<g, 256, 0, st>>>(n, x, d32, 1.0);
    LA_TRY(spmv_launch(S->Ap, -1.0, x, 1.0, r64, b, LA_F64, st));
    LA_TRY(dot(S, r64, r64, OP_STORE, st));
    double rr64;
    LA_TRY(read_scalar(S, S_DOT, &rr64, st));
    loc->rel_residual = std::sqrt(rr64) / bn;
    if (loc->rel_residual >= rtol)
      return LA_ERR_NOT_CONVERGED;
  }
  return LA_OK;
}

} // namespace

void pcg_destroy(la_pcg_t S);

la_status pcg_create(la_csr_t A, const int *u_ai, const int *u_aj,
                     const double *icc_av, la_pcg_mode mode, la_pcg_t *out) {
  auto *S = new la_pcg_s();
  S->A = A;
  S->mode = mode;
  const int n = S->n = A->n, base = A->base;
  auto fail = [&](la_status s) {
    pcg_destroy(S);
    return s;
  };
  // Preconditioner factors: strict U + diag, and strict L = U^T (same diag).
  const int unnz = u_ai[n] - base;
  bool lower = false; // an entry below the diagonal: not an IC factor
#pragma omp parallel for schedule(static) reduction(|| : lower)
  for (int i = 0; i < n; i++)
    for (int k = u_ai[i] - base; k < u_ai[i + 1] - base; k++)
      lower = lower || u_aj[k] - base < i;
  if (lower) {
    set_error("IC factor must be upper triangular");
    return fail(LA_ERR_INVALID_ARG);
  }
  // scratch left uninitialised: every entry is written before it is read
  const size_t m = std::max(unnz, 1);
  std::unique_ptr<int[]> s_aj(new int[m]), t_aj(new int[m]);
  std::unique_ptr<double[]> s_av(new double[m]), t_av(new double[m]);
  std::vector<int> l_ai(n + 1), l_aj(1), s_ai(n + 1), t_ai(n + 1);
  std::vector<double> l_av(1), d(n);
  int lnnz = 0, snnz = 0;
  split_ldu(n, base, u_ai, u_aj, icc_av, l_ai.data(), l_aj.data(), l_av.data(), d.data(),
            s_ai.data(), s_aj.get(), s_av.get(), &lnnz, &snnz);
  transpose(n, n, base, s_ai.data(), s_aj.get(), s_av.get(), t_ai.data(), t_aj.get(),
            t_av.get());
  const la_dtype fd = mode == LA_PCG_MIXED ? LA_F32 : LA_F64;
  la_status s;
  S->L = new la_trsv_plan_s();
  S->L->n = n;
  S->L->nnz = snnz;
  S->L->base = base;
  S->L->uplo = LA_LOWER;
  S->L->dtype = fd;
  S->L->unit = false;
  if ((s = trsv_build(S->L, t_ai.data(), t_aj.get(), t_av.get(), d.data())) != LA_OK)
    return fail(s);
  S->U = new la_trsv_plan_s();
  S->U->n = n;
  S->U->nnz = snnz;
  S->U->base = base;
  S->U->uplo = LA_UPPER;
  S->U->dtype = fd;
  S->U->unit = false;
  if ((s = trsv_build(S->U, s_ai.data(), s_aj.get(), s_av.get(), d.data())) != LA_OK)
    return fail(s);
  S->Ap = new la_spmv_plan_s();
  S->Ap->A = A;
  S->Ap->kind = LA_SPMV_SEGSUM;
  if ((s = spmv_plan_build(S->Ap)) != LA_OK)
    return fail(s);
  if (mode == LA_PCG_MIXED && A->av32.p == nullptr) {
    set_error("mixed PCG needs FP32 matrix values (create A with LA_CSR_KEEP_F32)");
    return fail(LA_ERR_INVALID_ARG);
  }
  const size_t v8 = sizeof(double) * std::max(n, 1), v4 = sizeof(float) * std::max(n, 1);
  for (DevBuf *b : {&S->r, &S->z, &S->p, &S->q, &S->t})
    if ((s = b->alloc(v8)) != LA_OK)
      return fail(s);
  if (mode == LA_PCG_MIXED)
    for (DevBuf *b : {&S->r32, &S->z32, &S->p32, &S->q32, &S->t32, &S->d32, &S->p32b})
      if ((s = b->alloc(v4)) != LA_OK)
        return fail(s);
  S->dot_blocks = std::max(1, std::min(2 * sm_count(), (n + kDotThreads - 1) / kDotThreads));
  if ((s = S->scal.alloc(sizeof(double) * S_COUNT)) != LA_OK ||
      (s = S->partials.alloc(sizeof(double) * 2 * S->dot_blocks)) != LA_OK ||
      (s = S->ticket.alloc(sizeof(unsigned))) != LA_OK ||
      (s = S->bar.alloc(sizeof(unsigned) * 4)) != LA_OK)
    return fail(s);
  // The fused kernels need every block resident at once (cooperative
  // launch); LA_PCG_FUSED=0 keeps the separate dot / update launches (same
  // iterates, bit for bit).
  if (const char *e = std::getenv("LA_PCG_RELIABLE_DELTA")) { // tuning override
    const double d = std::atof(e);
    if (d > 0.0 && d < 1.0)
      S->reliable_delta = d;
  }
  if (const char *e = std::getenv("LA_PCG_AHEAD_MARGIN")) { // tuning override
    const double m = std::atof(e);
    if (m >= 1.0)
      S->ahead_margin = m;
  }
  S->fused = true;
  if (const char *e = std::getenv("LA_PCG_FUSED"))
    S->fused = std::atoi(e) != 0;
  if (S->fused) {
    const void *fns[] = {(const void *)pcg_update_kernel<double>,
                         (const void *)pcg_update_kernel<float>};
    for (const void *f : fns) {
      int per_sm = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, f, kDotThreads, 0) !=
              cudaSuccess ||
          (long long)per_sm * sm_count() < S->dot_blocks) {
        cudaGetLastError();
        S->fused = false;
      }
    }
  }
  if (cudaMemset(S->bar.p, 0, S->bar.bytes) != cudaSuccess ||
      cudaMemset(S->ticket.p, 0, sizeof(unsigned)) != cudaSuccess ||
      cudaEventCreate(&S->ev0) != cudaSuccess || cudaEventCreate(&S->ev1) != cudaSuccess ||
      cudaEventCreateWithFlags(&S->ev_rr, cudaEventDisableTiming) != cudaSuccess ||
      cudaMallocHost((void **)&S->h_rr, sizeof(double)) != cudaSuccess) {
    set_error("PCG setup: CUDA error");
    return fail(LA_ERR_CUDA);
  }
  *out = S;
  return LA_OK;
}

la_status pcg_solve(la_pcg_t S, const double *b, double *x, double rtol,
                    int maxit, la_pcg_info *info, cudaStream_t st) {
  la_pcg_info loc{};
  la_status res = LA_OK;
  const int n = S->n;
  LA_CUDA_TRY(cudaEventRecord(S->ev0, st));
  // ||b||
  LA_TRY(dot(S, b, b, OP_STORE, st));
  double bb;
  LA_TRY(read_scalar(S, S_DOT, &bb, st));
  const double bn = std::sqrt(bb);
  if (bn == 0.0 || n == 0) {
    zero_kernel<<<vec_grid(n), 256, 0, st>>>(n, x);
    loc.outer_iterations = 1;
  } else if (S->mode == LA_PCG_FP64) {
    res = pcg_run<double>(S, b, x, S->r.as<double>(), S->z.as<double>(),
                          S->p.as<double>(), S->q.as<double>(), S->t.as<double>(),
                          LA_F64, rtol, maxit, b, bn, &loc.iterations,
                          &loc.rel_residual, st);
    loc.outer_iterations = 1;
  } else {
    res = pcg_mixed(S, b, x, bn, rtol, maxit, &loc, st);
  }
  LA_CUDA_TRY(cudaEventRecord(S->ev1, st));
  LA_CUDA_TRY(cudaEventSynchronize(S->ev1));
  float ms = 0;
  LA_CUDA_TRY(cudaEventElapsedTime(&ms, S->ev0, S->ev1));
  loc.solve_ms = ms;
  if (res == LA_OK) {
    LA_TRY(trsv_check(S->L, st));
    LA_TRY(trsv_check(S->U, st));
  }
  LA_TRY(barrier_check(S, st));
  if (info)
    *info = loc;
  if (res == LA_ERR_NOT_CONVERGED)
    set_error("PCG did not reach rtol %.3g in %d iterations (residual %.3g)",
              rtol, maxit, loc.rel_residual);
  return res;
}

// Adjoint of u = A^-1 b for a loss L(u): lambda = A^-T dL/du (A is
// symmetric, so one more PCG solve with the same operator and
// preconditioner), dL/db = lambda, dL/dA_ij = -lambda_i u_j over A's stored
// pattern (the sampled outer product of la_sddmm_pattern).
la_status sddmm_launch(la_spmv_plan_t P, double alpha, const double *g,
                       const double *x, double *dv, cudaStream_t st);

la_status pcg_adjoint(la_pcg_t S, const double *g, const double *u, double *dl_db,
                      double *dl_dv, double rtol, int maxit, la_pcg_info *info,
                      cudaStream_t st) {
  LA_TRY(pcg_solve(S, g, dl_db, rtol, maxit, info, st));
  if (dl_dv)
    LA_TRY(sddmm_launch(S->Ap, -1.0, dl_db, u, dl_dv, st));
  return LA_OK;
}

void pcg_destroy(la_pcg_t S) {
  if (!S)
    return;
  if (S->ev0)
    cudaEventDestroy(S->ev0);
  if (S->ev1)
    cudaEventDestroy(S->ev1);
  if (S->ev_rr)
    cudaEventDestroy(S->ev_rr);
  if (S->h_rr)
    cudaFreeHost(S->h_rr);
  delete S->L;
  delete S->U;
  delete S->Ap;
  delete S;
}

} // namespace la
