// la_capi.cu -- the extern "C" boundary (include/la_b200.h).
#include "la_internal.h"

#include <cstdarg>
#include <cstring>
#include <memory>
#include <mutex>

namespace la {

la_status spmv_launch(la_spmv_plan_t P, double alpha, const void *x,
                      double beta, void *y, const void *yin, la_dtype vd,
                      cudaStream_t st);
la_status spmv_xparts_launch(la_spmv_plan_t P, double alpha, const void *const *xparts,
                             const int *part_start, int nparts, double beta, void *y,
                             la_dtype vd, cudaStream_t st);
la_status sddmm_launch(la_spmv_plan_t P, double alpha, const double *g,
                       const double *x, double *dv, cudaStream_t st);
la_status spmv_ceiling_launch(la_spmv_plan_t P, const double *x, int gather, double *sink,
                              cudaStream_t st);
la_status spmv_noalloc(la_spmv_kind kind, int n, int nnz, int base, const int *ai,
                       const int *aj, const double *av, double alpha, const double *x,
                       double beta, double *y, cudaStream_t st);
la_status spmv_plan_build(la_spmv_plan_t P);
la_status spmv_host_chunked(la_spmv_plan_t P, double alpha, const double *x, double beta,
                            double *y);
la_status trsv_launch(la_trsv_plan_t P, const void *b, void *x,
                      cudaStream_t st);
la_status trsv_build(la_trsv_plan_t P, const int *ai, const int *aj,
                     const double *av, const double *diag, const int *iperm = nullptr,
                     const int *prefix = nullptr, int nlevels = 0);
la_status trsv_check(la_trsv_plan_t P, cudaStream_t st);
la_status pcg_create(la_csr_t A, const int *u_ai, const int *u_aj,
                     const double *icc_av, la_pcg_mode mode, la_pcg_t *out);
la_status pcg_solve(la_pcg_t S, const double *b, double *x, double rtol,
                    int maxit, la_pcg_info *info, cudaStream_t st);
void pcg_destroy(la_pcg_t S);
la_status pcg_adjoint(la_pcg_t S, const double *g, const double *u, double *dl_db,
                      double *dl_dv, double rtol, int maxit, la_pcg_info *info,
                      cudaStream_t st);

namespace {
thread_local char g_err[512] = "";

__global__ void f64_to_f32_kernel(long n, const double *in, float *out) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x)
    out[i] = float(in[i]);
}
} // namespace

void set_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(g_err, sizeof g_err, fmt, ap);
  va_end(ap);
}
const char *get_error() { return g_err; }

la_status require_device() {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    set_error("no CUDA device: %s", cudaGetErrorString(e));
    return LA_ERR_NO_DEVICE;
  }
  int major = 0;
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
  if (major != 10) {
    set_error("device %d has compute capability %d.x; this library is built "
              "for sm_100a (B200)", dev, major);
    return LA_ERR_NO_DEVICE;
  }
  return LA_OK;
}

int sm_count() {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms > 0 ? sms : 1;
}

// Every device buffer is allocated kPad bytes longer than asked, so that
// 16-byte-granular bulk copies of a ragged tail never leave the allocation.
constexpr size_t kPad = 64;

la_status DevBuf::alloc(size_t b) {
  release();
  cudaError_t e = cudaMalloc(&p, b + kPad);
  if (e != cudaSuccess) {
    p = nullptr;
    set_error("cudaMalloc(%zu) failed: %s", b, cudaGetErrorString(e));
    return LA_ERR_ALLOC;
  }
  bytes = b;
  return LA_OK;
}
// Large uploads (plans and matrices, built in pageable host memory) go
// through two pinned halves of a staging area: the host's threads copy one
// chunk into a half while the previous chunk crosses PCIe from the other.
// Pageable cudaMemcpy measured ~6.6 GB/s on the B200 hosts.  One staging
// area per process, behind a mutex, with its stream on the device current at
// its first use; uploads while another device is current, or when it cannot
// be pinned, or a copy that fails part-way, take the plain copy.
namespace {
constexpr size_t kStageChunk = size_t(16) << 20, kStageMin = size_t(8) << 20;
std::mutex g_stage_mu;
char *g_stage = nullptr; // 2 x kStageChunk, pinned
cudaStream_t g_stage_stream = nullptr;
cudaEvent_t g_stage_done[2] = {nullptr, nullptr};
bool g_stage_failed = false;
int g_stage_dev = -1;

bool stage_ready() {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess)
    return false;
  if (g_stage)
    return dev == g_stage_dev;
  if (g_stage_failed)
    return false;
  g_stage_dev = dev;
  if (cudaHostAlloc(&g_stage, 2 * kStageChunk, cudaHostAllocDefault) != cudaSuccess ||
      cudaStreamCreateWithFlags(&g_stage_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&g_stage_done[0], cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&g_stage_done[1], cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    g_stage = nullptr;
    g_stage_failed = true;
    return false;
  }
  return true;
}

bool staged_upload(void *dst, const void *src, size_t b) {
  std::lock_guard<std::mutex> lock(g_stage_mu);
  if (!stage_ready())
    return false;
  for (size_t off = 0, k = 0; off < b; off += kStageChunk, k++) {
    const int h = (int)(k & 1);
    const size_t len = std::min(kStageChunk, b - off);
    char *stage = g_stage + h * kStageChunk;
    if (k >= 2 && cudaEventSynchronize(g_stage_done[h]) != cudaSuccess)
      return false;
    constexpr size_t kPiece = size_t(1) << 20;
    const long long pieces = (long long)((len + kPiece - 1) / kPiece);
#pragma omp parallel for schedule(static)
    for (long long q = 0; q < pieces; q++) {
      const size_t o = (size_t)q * kPiece;
      std::memcpy(stage + o, static_cast<const char *>(src) + off + o, std::min(kPiece, len - o));
    }
    if (cudaMemcpyAsync(static_cast<char *>(dst) + off, stage, len, cudaMemcpyHostToDevice,
                        g_stage_stream) != cudaSuccess ||
        cudaEventRecord(g_stage_done[h], g_stage_stream) != cudaSuccess)
      return false;
  }
  return cudaStreamSynchronize(g_stage_stream) == cudaSuccess;
}
} // namespace

la_status DevBuf::upload(const void *host, size_t b) {
  LA_TRY(alloc(b));
  if (!host || !b)
    return LA_OK;
  if (b >= kStageMin && staged_upload(p, host, b))
    return LA_OK;
  cudaGetLastError();
  LA_CUDA_TRY(cudaMemcpy(p, host, b, cudaMemcpyHostToDevice));
  return LA_OK;
}
void DevBuf::release() {
  if (p)
    cudaFree(p);
  p = nullptr;
  bytes = 0;
}

} // namespace la

const void *la_csr_s::values(la_dtype vd) const {
  if (vd == dtype)
    return av.p;
  if (vd == LA_F32 && av32.p)
    return av32.p;
  return nullptr;
}

using namespace la;

static cudaStream_t S(la_stream_t s) { return static_cast<cudaStream_t>(s); }

namespace la {
// The optional FP32 copy of an FP64 matrix's values (LA_CSR_KEEP_F32).
la_status csr_finish(la_csr_t A, int flags) {
  if ((flags & LA_CSR_KEEP_F32) && A->dtype == LA_F64 && A->nnz > 0) {
    LA_TRY(A->av32.alloc(sizeof(float) * A->nnz));
    f64_to_f32_kernel<<<std::min((A->nnz + 255) / 256, 8192), 256>>>(
        A->nnz, A->av.as<double>(), A->av32.as<float>());
    LA_CUDA_TRY(cudaGetLastError());
    LA_CUDA_TRY(cudaDeviceSynchronize());
  }
  return LA_OK;
}
} // namespace la

extern "C" {

const char *la_last_error_string(void) { return la::get_error(); }
const char *la_version(void) { return "linearalgebra_b200 0.1 (sm_100a)"; }

la_status la_device_sm_count(int *sms) {
  LA_CHECK_ARG(sms, "sms is NULL");
  LA_TRY(require_device());
  *sms = sm_count();
  return LA_OK;
}

// ------------------------------------------------------------------ CSR

la_status la_csr_create(int n, int ncols, int base, const int *ai,
                        const int *aj, const void *av, la_dtype dtype,
                        int flags, la_csr_t *out) {
  LA_CHECK_ARG(out && ai && n >= 0 && ncols >= 0, "null pointer or size");
  LA_CHECK_ARG(base == 0 || base == 1, "base must be 0 or 1");
  LA_CHECK_ARG(dtype == LA_F64 || dtype == LA_F32, "dtype");
  const long nnzl = (long)ai[n] - base;
  LA_CHECK_ARG(nnzl >= 0 && nnzl < (1L << 31), "nnz out of int32 range");
  LA_CHECK_ARG(nnzl == 0 || (aj && av), "aj/av NULL with nnz > 0");
  std::string why;
  if (!valid_csr(n, ncols, base, ai, aj, &why)) {
    set_error("invalid CSR: %s", why.c_str());
    return LA_ERR_BAD_CSR;
  }
  LA_TRY(require_device());
  std::unique_ptr<la_csr_s> A(new la_csr_s());
  A->n = n;
  A->ncols = ncols;
  A->nnz = (int)nnzl;
  A->base = base;
  A->dtype = dtype;
  A->h_ai.assign(ai, ai + n + 1);
  LA_TRY(A->ai.upload(ai, sizeof(int) * (n + 1)));
  LA_TRY(A->aj.upload(aj, sizeof(int) * A->nnz));
  LA_TRY(A->av.upload(av, (dtype == LA_F64 ? 8 : 4) * (size_t)A->nnz));
  LA_TRY(csr_finish(A.get(), flags));
  *out = A.release();
  return LA_OK;
}

la_status la_csr_create_device(int n, int ncols, int nnz, int base,
                               const int *d_ai, const int *d_aj,
                               const void *d_av, la_dtype dtype, int flags,
                               la_csr_t *out) {
  LA_CHECK_ARG(out && d_ai && n >= 0 && ncols >= 0 && nnz >= 0, "arguments");
  LA_CHECK_ARG(base == 0 || base == 1, "base must be 0 or 1");
  LA_TRY(require_device());
  std::unique_ptr<la_csr_s> A(new la_csr_s());
  A->n = n;
  A->ncols = ncols;
  A->nnz = nnz;
  A->base = base;
  A->dtype = dtype;
  A->h_ai.resize(n + 1);
  LA_CUDA_TRY(cudaMemcpy(A->h_ai.data(), d_ai, sizeof(int) * (n + 1),
                         cudaMemcpyDeviceToHost));
  if (A->h_ai[0] != base || A->h_ai[n] - base != nnz) {
    set_error("invalid CSR: ai[0] != base or ai[n] - base != nnz");
    return LA_ERR_BAD_CSR;
  }
  const size_t vs = dtype == LA_F64 ? 8 : 4;
  LA_TRY(A->ai.alloc(sizeof(int) * (n + 1)));
  LA_TRY(A->aj.alloc(sizeof(int) * nnz));
  LA_TRY(A->av.alloc(vs * nnz));
  LA_CUDA_TRY(cudaMemcpy(A->ai.p, d_ai, sizeof(int) * (n + 1), cudaMemcpyDeviceToDevice));
  if (nnz) {
    LA_CUDA_TRY(cudaMemcpy(A->aj.p, d_aj, sizeof(int) * nnz, cudaMemcpyDeviceToDevice));
    LA_CUDA_TRY(cudaMemcpy(A->av.p, d_av, vs * nnz, cudaMemcpyDeviceToDevice));
  }
  LA_TRY(csr_finish(A.get(), flags));
  *out = A.release();
  return LA_OK;
}

la_status la_csr_update_values(la_csr_t A, const void *av, int on_device) {
  LA_CHECK_ARG(A && (av || A->nnz == 0), "arguments");
  const size_t vs = A->dtype == LA_F64 ? 8 : 4;
  if (A->nnz)
    LA_CUDA_TRY(cudaMemcpy(A->av.p, av, vs * A->nnz,
                           on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice));
  if (A->av32.p)
    LA_TRY(csr_finish(A, LA_CSR_KEEP_F32));
  return LA_OK;
}

la_status la_csr_info(la_csr_t A, int *n, int *ncols, int *nnz, int *base,
                      la_dtype *dtype) {
  LA_CHECK_ARG(A, "A is NULL");
  if (n) *n = A->n;
  if (ncols) *ncols = A->ncols;
  if (nnz) *nnz = A->nnz;
  if (base) *base = A->base;
  if (dtype) *dtype = A->dtype;
  return LA_OK;
}

la_status la_csr_destroy(la_csr_t A) {
  delete A;
  return LA_OK;
}

la_status la_csr_download(la_csr_t A, int *ai, int *aj, void *av) {
  LA_CHECK_ARG(A, "A is NULL");
  if (ai)
    LA_CUDA_TRY(cudaMemcpy(ai, A->ai.p, sizeof(int) * (A->n + 1), cudaMemcpyDeviceToHost));
  if (aj && A->nnz)
    LA_CUDA_TRY(cudaMemcpy(aj, A->aj.p, sizeof(int) * A->nnz, cudaMemcpyDeviceToHost));
  if (av && A->nnz)
    LA_CUDA_TRY(cudaMemcpy(av, A->av.p, (A->dtype == LA_F64 ? 8 : 4) * (size_t)A->nnz,
                           cudaMemcpyDeviceToHost));
  return LA_OK;
}

// ------------------------------------------------------------------ ingest
la_status la_csr_from_coo(int nrows, int ncols, long long nnz, int base, const int *rows,
                          const int *cols, const void *vals, la_dtype dtype, int flags,
                          la_csr_t *out) {
  LA_CHECK_ARG(out && nrows >= 0 && ncols >= 0, "arguments");
  LA_CHECK_ARG(base == 0 || base == 1, "base must be 0 or 1");
  LA_CHECK_ARG(dtype == LA_F64 || dtype == LA_F32, "dtype");
  LA_CHECK_ARG(nnz >= 0 && nnz < (1LL << 31), "nnz out of int32 range");
  LA_CHECK_ARG(nnz == 0 || (rows && cols && vals), "rows/cols/vals NULL with nnz > 0");
  return csr_from_coo(nrows, ncols, nnz, base, rows, cols, vals, dtype, flags, out);
}

// Two-call pattern of the host readers: with rows == NULL only the sizes
// are returned; then arrays of *nnz entries are filled.
static la_status copy_coo(const std::vector<int> &r, const std::vector<int> &c,
                          const std::vector<double> &v, long long *nnz, int *rows, int *cols,
                          double *vals) {
  if (rows || cols || vals) {
    LA_CHECK_ARG(rows && cols && vals, "rows/cols/vals: all or none");
    LA_CHECK_ARG(*nnz >= (long long)r.size(), "arrays shorter than the entry count");
    std::memcpy(rows, r.data(), sizeof(int) * r.size());
    std::memcpy(cols, c.data(), sizeof(int) * c.size());
    std::memcpy(vals, v.data(), sizeof(double) * v.size());
  }
  *nnz = (long long)r.size();
  return LA_OK;
}

la_status la_read_binary_coo(const char *path, int base, long long *nnz, int *rows, int *cols,
                             double *vals, int *m, int *n) {
  LA_CHECK_ARG(path && nnz && m && n && (base == 0 || base == 1), "arguments");
  std::vector<int> r, c;
  std::vector<double> v;
  LA_TRY(read_binary_coo(path, base, r, c, v, m, n));
  return copy_coo(r, c, v, nnz, rows, cols, vals);
}

la_status la_read_matrix_market(const char *path, long long *nnz, int *rows, int *cols,
                                double *vals, int *m, int *n) {
  LA_CHECK_ARG(path && nnz && m && n, "arguments");
  std::string text;
  LA_TRY(read_file(path, text));
  std::vector<int> r, c;
  std::vector<double> v;
  LA_TRY(parse_matrix_market(text.data(), text.size(), r, c, v, m, n));
  return copy_coo(r, c, v, nnz, rows, cols, vals);
}

la_status la_csr_read_binary_coo(const char *path, int base, int flags, la_csr_t *out) {
  LA_CHECK_ARG(path && out && (base == 0 || base == 1), "arguments");
  std::vector<int> r, c;
  std::vector<double> v;
  int m = 0, n = 0;
  LA_TRY(read_binary_coo(path, base, r, c, v, &m, &n));
  return csr_from_coo(m, n, (long long)r.size(), base, r.data(), c.data(), v.data(), LA_F64,
                      flags, out);
}

la_status la_csr_parse_matrix_market(const char *text, size_t len, int flags, la_csr_t *out) {
  LA_CHECK_ARG(text && out, "arguments");
  std::vector<int> r, c;
  std::vector<double> v;
  int m = 0, n = 0;
  LA_TRY(parse_matrix_market(text, len, r, c, v, &m, &n));
  return csr_from_coo(m, n, (long long)r.size(), 0, r.data(), c.data(), v.data(), LA_F64, flags,
                      out);
}

la_status la_csr_read_matrix_market(const char *path, int flags, la_csr_t *out) {
  LA_CHECK_ARG(path && out, "arguments");
  std::string text;
  LA_TRY(read_file(path, text));
  return la_csr_parse_matrix_market(text.data(), text.size(), flags, out);
}

// ----------------------------------------------------------------- SpMV
la_status la_spmv_plan_create(la_csr_t A, la_spmv_kind kind,
                              la_spmv_plan_t *out) {
  LA_CHECK_ARG(A && out, "arguments");
  LA_CHECK_ARG(kind == LA_SPMV_SEGSUM || kind == LA_SPMV_ALBUS, "kind");
  std::unique_ptr<la_spmv_plan_s> P(new la_spmv_plan_s());
  P->A = A;
  P->kind = kind;
  LA_TRY(spmv_plan_build(P.get()));
  *out = P.release();
  return LA_OK;
}

la_status la_spmv(la_spmv_plan_t plan, double alpha, const void *x,
                  double beta, void *y, la_dtype vdtype, la_stream_t stream) {
  LA_CHECK_ARG(plan && (x || plan->A->n == 0) && (y || plan->A->n == 0), "arguments");
  LA_CHECK_ARG(x != y || plan->A->n == 0, "x and y must not alias");
  return spmv_launch(plan, alpha, x, beta, y, y, vdtype, S(stream));
}

la_status la_spmv_host(la_spmv_plan_t plan, double alpha, const double *x,
                       double beta, double *y) {
  LA_CHECK_ARG(plan && x && y, "arguments");
  return spmv_host_chunked(plan, alpha, x, beta, y);
}

la_status la_spmv_layout(la_spmv_plan_t plan, int *row_slots) {
  LA_CHECK_ARG(plan && row_slots, "arguments");
  *row_slots = plan->ell_k;
  return LA_OK;
}

la_status la_spmv_plan_destroy(la_spmv_plan_t plan) {
  if (plan) {
    delete plan->Atplan;
    delete plan->At;
  }
  delete plan;
  return LA_OK;
}

static la_status ensure_transpose(la_spmv_plan_t P) {
  if (P->Atplan)
    return LA_OK;
  const la_csr_t A = P->A;
  if (A->dtype != LA_F64) {
    set_error("adjoint needs an FP64 matrix");
    return LA_ERR_INVALID_ARG;
  }
  std::vector<int> aj(std::max(A->nnz, 1)), tai(A->ncols + 1), taj(std::max(A->nnz, 1));
  std::vector<double> av(std::max(A->nnz, 1)), tav(std::max(A->nnz, 1));
  if (A->nnz) {
    LA_CUDA_TRY(cudaMemcpy(aj.data(), A->aj.p, sizeof(int) * A->nnz, cudaMemcpyDeviceToHost));
    LA_CUDA_TRY(cudaMemcpy(av.data(), A->av.p, sizeof(double) * A->nnz, cudaMemcpyDeviceToHost));
  }
  transpose(A->n, A->ncols, A->base, A->h_ai.data(), aj.data(), av.data(),
            tai.data(), taj.data(), tav.data());
  std::unique_ptr<la_csr_s> T(new la_csr_s());
  T->n = A->ncols;
  T->ncols = A->n;
  T->nnz = A->nnz;
  T->base = A->base;
  T->dtype = LA_F64;
  T->h_ai = tai;
  LA_TRY(T->ai.upload(tai.data(), sizeof(int) * tai.size()));
  LA_TRY(T->aj.upload(taj.data(), sizeof(int) * A->nnz));
  LA_TRY(T->av.upload(tav.data(), sizeof(double) * A->nnz));
  std::unique_ptr<la_spmv_plan_s> TP(new la_spmv_plan_s());
  TP->A = T.get();
  TP->kind = P->kind;
  LA_TRY(spmv_plan_build(TP.get()));
  P->At = T.release();
  P->Atplan = TP.release();
  return LA_OK;
}

la_status la_spmv_transpose(la_spmv_plan_t plan, double alpha, const double *g,
                            double beta, double *out, la_stream_t stream) {
  LA_CHECK_ARG(plan && g && out && g != out, "arguments");
  LA_TRY(ensure_transpose(plan));
  return spmv_launch(plan->Atplan, alpha, g, beta, out, out, LA_F64, S(stream));
}

la_status la_spmv_xparts(la_spmv_plan_t plan, double alpha, const void *const *xparts,
                         const int *part_start, int nparts, double beta, void *y,
                         la_dtype vector_dtype, la_stream_t stream) {
  LA_CHECK_ARG(plan && xparts && part_start && (y || plan->A->n == 0), "arguments");
  LA_CHECK_ARG(nparts >= 1 && nparts <= LA_SPMV_MAX_XPARTS, "nparts out of range");
  LA_CHECK_ARG(part_start[0] == 0 && part_start[nparts] == plan->A->ncols,
               "part_start must run from 0 to the column count");
  for (int r = 0; r < nparts; r++) {
    LA_CHECK_ARG(part_start[r] <= part_start[r + 1], "part_start must not decrease");
    LA_CHECK_ARG(xparts[r] || part_start[r] == part_start[r + 1], "missing x slice");
  }
  LA_CHECK_ARG(vector_dtype == LA_F64 || vector_dtype == LA_F32, "vector dtype");
  return spmv_xparts_launch(plan, alpha, xparts, part_start, nparts, beta, y, vector_dtype,
                            S(stream));
}

la_status la_spmv_noalloc(la_spmv_kind kind, int n, int nnz, int base,
                          const int *d_ai, const int *d_aj, const double *d_av,
                          double alpha, const double *d_x, double beta, double *d_y,
                          la_stream_t stream) {
  LA_CHECK_ARG(n >= 0 && nnz >= 0 && (base == 0 || base == 1), "sizes / base");
  LA_CHECK_ARG(kind == LA_SPMV_SEGSUM || kind == LA_SPMV_ALBUS, "kind");
  LA_CHECK_ARG(n == 0 || (d_ai && d_x && d_y && d_x != d_y), "pointers");
  LA_CHECK_ARG(nnz == 0 || (d_aj && d_av), "aj / av");
  return spmv_noalloc(kind, n, nnz, base, d_ai, d_aj, d_av, alpha, d_x, beta, d_y,
                      S(stream));
}

la_status la_spmv_ceiling(la_spmv_plan_t plan, const double *x, int gather, double *sink,
                          la_stream_t stream) {
  LA_CHECK_ARG(plan && sink && (!gather || x), "arguments");
  return spmv_ceiling_launch(plan, x, gather, sink, S(stream));
}

la_status la_sddmm_pattern(la_spmv_plan_t plan, double alpha, const double *g,
                           const double *x, double *dv, la_stream_t stream) {
  LA_CHECK_ARG(plan && g && x && (dv || plan->A->nnz == 0), "arguments");
  return sddmm_launch(plan, alpha, g, x, dv, S(stream));
}

// ------------------------------------------------------- host analysis
la_status la_topological_sort2(la_uplo uplo, int n, int base, const int *ai,
                               const int *aj, int *iperm, int *prefix,
                               int *levels) {
  LA_CHECK_ARG(ai && iperm && prefix && levels && n >= 0, "arguments");
  *levels = n == 0 ? 0 : topological_sort2(uplo, n, base, ai, aj, iperm, prefix);
  if (n == 0)
    prefix[0] = 0;
  return LA_OK;
}

la_status la_topological_sort2_device(la_uplo uplo, int n, int base, const int *ai,
                                      const int *aj, int *iperm, int *prefix, int *levels) {
  LA_CHECK_ARG(ai && iperm && prefix && levels && n >= 0, "arguments");
  LA_CHECK_ARG(base == 0 || base == 1, "base must be 0 or 1");
  LA_CHECK_ARG(n == 0 || ai[n] - base == 0 || aj, "aj");
  if (n == 0) {
    *levels = 0;
    prefix[0] = 0;
    return LA_OK;
  }
  LA_TRY(require_device());
  return topological_sort2_device(uplo, n, base, ai, aj, iperm, prefix, levels);
}

la_status la_topological_sort(la_uplo uplo, int n, int base, const int *ai, const int *aj,
                              int *iperm, int *prefix, int *result) {
  LA_CHECK_ARG(ai && iperm && prefix && result && n >= 0, "arguments");
  LA_CHECK_ARG(uplo == LA_LOWER || uplo == LA_UPPER, "uplo");
  std::string why;
  if (!valid_csr(n, n, base, ai, aj, &why)) {
    set_error("invalid CSR: %s", why.c_str());
    return LA_ERR_BAD_CSR;
  }
  const int r = topological_sort_kahn(uplo, n, base, ai, aj, iperm, prefix);
  if (r < 0) {
    set_error("la_topological_sort: the dependencies form a cycle");
    return LA_ERR_INVALID_ARG;
  }
  *result = r;
  return LA_OK;
}

la_status la_rcm(int n, int base, const int *ai, const int *aj, int *iperm,
                 int *perm) {
  LA_CHECK_ARG(ai && iperm && perm && n >= 0, "arguments");
  // SerialCM walks out-edges from its BFS source; on a structurally
  // unsymmetric pattern the reference reads unfilled ordering slots
  // (reordering/Reordering.cpp:96-107), so such input is rejected here.
  const int nnz = ai[n] - base;
  std::vector<int> tai(n + 1), taj(std::max(nnz, 1));
  transpose(n, n, base, ai, aj, nullptr, tai.data(), taj.data(), nullptr);
  if (std::memcmp(tai.data(), ai, sizeof(int) * (n + 1)) != 0 ||
      std::memcmp(taj.data(), aj, sizeof(int) * nnz) != 0) {
    set_error("la_rcm needs a structurally symmetric pattern");
    return LA_ERR_INVALID_ARG;
  }
  return rcm(n, base, ai, aj, iperm, perm);
}

la_status la_rcm_device(int n, int base, const int *ai, const int *aj, int *iperm,
                        int *perm) {
  LA_CHECK_ARG(ai && iperm && perm && n >= 0 && (base == 0 || base == 1), "arguments");
  LA_CHECK_ARG(ai[n] - base == 0 || aj, "aj");
  if (n == 0)
    return LA_OK;
  LA_TRY(require_device());
  bool handled = false; // pattern checked on the device; connected: ordered there too
  LA_TRY(rcm_device_connected(n, base, ai, aj, iperm, perm, &handled));
  if (handled)
    return LA_OK;
  return rcm(n, base, ai, aj, iperm, perm, true);
}

la_status la_permute(int n, int base, const int *ai, const int *aj,
                     const double *av, const int *iperm, const int *perm,
                     int *p_ai, int *p_aj, double *p_av) {
  LA_CHECK_ARG(ai && aj && av && p_ai && p_aj && p_av && n >= 0, "arguments");
  permute(n, base, ai, aj, av, iperm, perm, p_ai, p_aj, p_av);
  return LA_OK;
}

la_status la_ilu0(int n, int base, const int *ai, const int *aj, const double *av,
                  double *lu_av) {
  LA_CHECK_ARG(ai && aj && av && lu_av && n >= 0, "arguments");
  std::string why;
  if (!valid_csr(n, n, base, ai, aj, &why)) {
    set_error("invalid CSR: %s", why.c_str());
    return LA_ERR_BAD_CSR;
  }
  const int r = ilu0(n, base, ai, aj, av, lu_av);
  if (r == -2) {
    set_error("la_ilu0: a row has no diagonal entry");
    return LA_ERR_INVALID_ARG;
  }
  if (r >= 0) {
    set_error("la_ilu0: zero pivot in row %d", r);
    return LA_ERR_BREAKDOWN;
  }
  return LA_OK;
}

la_status la_permute_vec(int n, int base, const double *v, const int *iperm, double *out) {
  LA_CHECK_ARG(v && out && n >= 0, "arguments");
  permute_vec(n, base, v, iperm, out);
  return LA_OK;
}

la_status la_inverse_permute(int n, int base, const int *perm, int *iperm) {
  LA_CHECK_ARG(perm && iperm && n >= 0, "arguments");
  std::vector<char> seen(n, 0);
  for (int i = 0; i < n; i++) {
    const int p = perm[i] - base;
    LA_CHECK_ARG(p >= 0 && p < n && !seen[p], "perm must be a permutation");
    seen[p] = 1;
  }
  inverse_permute(n, base, perm, iperm);
  return LA_OK;
}

la_status la_diagonal(int n, int base, const int *ai, const int *aj, const double *av,
                      int *diagpos, double *diag, int invert, int *all_present) {
  LA_CHECK_ARG(ai && (aj || ai[n] == base) && (av || !diag) && n >= 0, "arguments");
  std::string why;
  if (!valid_csr(n, n, base, ai, aj, &why)) {
    set_error("invalid CSR: %s", why.c_str());
    return LA_ERR_BAD_CSR;
  }
  const bool all = diagonal(n, base, ai, aj, av, diagpos, diag, invert != 0);
  if (all_present)
    *all_present = all ? 1 : 0;
  return LA_OK;
}

la_status la_transpose(int rows, int cols, int base, const int *ai,
                       const int *aj, const double *av, int *t_ai, int *t_aj,
                       double *t_av) {
  LA_CHECK_ARG(ai && t_ai && (aj || ai[rows] == base) && rows >= 0, "arguments");
  transpose(rows, cols, base, ai, aj, av, t_ai, t_aj, t_av);
  return LA_OK;
}

la_status la_split_ldu(int n, int base, const int *ai, const int *aj,
                       const double *av, int *l_ai, int *l_aj, double *l_av,
                       double *d, int *u_ai, int *u_aj, double *u_av,
                       int *lnnz, int *unnz) {
  LA_CHECK_ARG(ai && l_ai && u_ai && d && lnnz && unnz && n >= 0, "arguments");
  split_ldu(n, base, ai, aj, av, l_ai, l_aj, l_av, d, u_ai, u_aj, u_av, lnnz, unnz);
  return LA_OK;
}

la_status la_split_triangle(la_uplo uplo, int n, int base, const int *ai,
                            const int *aj, const double *av, int *t_ai,
                            int *t_aj, double *t_av, int *tnnz) {
  LA_CHECK_ARG(ai && t_ai && tnnz && n >= 0, "arguments");
  *tnnz = split_triangle(uplo, n, base, ai, aj, av, t_ai, t_aj, t_av);
  return LA_OK;
}

la_status la_valid_csr(int rows, int cols, int base, const int *ai,
                       const int *aj) {
  LA_CHECK_ARG(ai, "ai is NULL");
  std::string why;
  if (!valid_csr(rows, cols, base, ai, aj, &why)) {
    set_error("invalid CSR: %s", why.c_str());
    return LA_ERR_BAD_CSR;
  }
  return LA_OK;
}

la_status la_icc0(int n, int base, const int *u_ai, const int *u_aj,
                  const double *u_av, double omega, double *icc_av) {
  LA_CHECK_ARG(u_ai && u_aj && u_av && icc_av && n >= 0, "arguments");
  for (int i = 0; i < n; i++)
    if (u_ai[i + 1] == u_ai[i] || u_aj[u_ai[i] - base] - base != i) {
      set_error("IC(0): row %d of the upper triangle does not start with its "
                "diagonal", i);
      return LA_ERR_INVALID_ARG;
    }
  if (!icc0(n, base, u_ai, u_aj, u_av, omega, icc_av)) {
    set_error("IC(0) breakdown: negative pivot (omega = %g)", omega);
    return LA_ERR_BREAKDOWN;
  }
  return LA_OK;
}

la_status la_icc0_shifted(int n, int base, const int *u_ai, const int *u_aj,
                          const double *u_av, double *icc_av,
                          double *shift_used) {
  double shift = 0.0;
  for (int restart = 0;; restart++) {
    const la_status s = la_icc0(n, base, u_ai, u_aj, u_av, shift, icc_av);
    if (s != LA_ERR_BREAKDOWN) {
      if (shift_used)
        *shift_used = shift;
      return s;
    }
    if (restart + 1 > 20) // _nrestart (incomplete_cholesky.h:28)
      return s;
    shift = std::max(2 * shift, 1e-3); // _initial_shift (incomplete_cholesky.h:27)
  }
}

// ------------------------------------------------ device factorisation
la_status la_icc0_plan_create(int n, int base, const int *u_ai, const int *u_aj,
                              la_factor_plan_t *out) {
  LA_CHECK_ARG(u_ai && out && n >= 0 && (base == 0 || base == 1), "arguments");
  LA_CHECK_ARG(u_ai[n] - base == 0 || u_aj, "u_aj");
  for (int i = 0; i < n; i++) {
    if (u_ai[i + 1] <= u_ai[i] || u_aj[u_ai[i] - base] - base != i) {
      set_error("IC(0): row %d of the upper triangle does not start with its diagonal", i);
      return LA_ERR_INVALID_ARG;
    }
    // the symbolic pass orders updates by walking rows backwards from a
    // column: columns must ascend strictly and stay below n
    for (int k = u_ai[i] - base + 1; k < u_ai[i + 1] - base; k++)
      if (u_aj[k] <= u_aj[k - 1] || u_aj[k] - base >= n) {
        set_error("IC(0): row %d of the upper triangle is not sorted within [%d, %d)", i, i, n);
        return LA_ERR_INVALID_ARG;
      }
  }
  LA_TRY(require_device());
  return factor_plan_create(0, n, base, u_ai, u_aj, out);
}

la_status la_ilu0_plan_create(int n, int base, const int *ai, const int *aj,
                              la_factor_plan_t *out) {
  LA_CHECK_ARG(ai && out && n >= 0 && (base == 0 || base == 1), "arguments");
  std::string why;
  if (!valid_csr(n, n, base, ai, aj, &why)) {
    set_error("invalid CSR: %s", why.c_str());
    return LA_ERR_BAD_CSR;
  }
  LA_TRY(require_device());
  return factor_plan_create(1, n, base, ai, aj, out);
}

la_status la_factor_numeric(la_factor_plan_t plan, const double *av, double omega,
                            double *out, int on_device, int *bad_row, la_stream_t stream) {
  LA_CHECK_ARG(plan && (plan->nnz == 0 || (av && out)), "arguments");
  int bad = -1;
  const la_status s = factor_numeric(plan, av, omega, out, on_device != 0, &bad, S(stream));
  if (bad_row)
    *bad_row = bad;
  return s;
}

la_status la_factor_icc0_shifted(la_factor_plan_t plan, const double *av, double *out,
                                 int on_device, double *shift_used, la_stream_t stream) {
  LA_CHECK_ARG(plan && plan->kind == 0, "an IC(0) plan");
  double shift = 0.0;
  for (int restart = 0;; restart++) {
    int bad = -1;
    const la_status s = factor_numeric(plan, av, shift, out, on_device != 0, &bad, S(stream));
    if (s != LA_ERR_BREAKDOWN) {
      if (shift_used)
        *shift_used = shift;
      return s;
    }
    if (restart + 1 > 20) // _nrestart (incomplete_cholesky.h:28)
      return s;
    shift = std::max(2 * shift, 1e-3); // _initial_shift (incomplete_cholesky.h:27)
  }
}

la_status la_factor_levels(la_factor_plan_t plan, int *levels) {
  LA_CHECK_ARG(plan && levels, "arguments");
  *levels = plan->levels;
  return LA_OK;
}

la_status la_factor_plan_destroy(la_factor_plan_t plan) {
  delete plan;
  return LA_OK;
}

// ------------------------------------------------------------------ trsv
// A valid CSR whose entries all lie in the strict `uplo` triangle.
static la_status check_strict_triangle(la_uplo uplo, int n, int base, const int *ai,
                                       const int *aj) {
  std::string why;
  if (!valid_csr(n, n, base, ai, aj, &why)) {
    set_error("invalid CSR: %s", why.c_str());
    return LA_ERR_BAD_CSR;
  }
  for (int i = 0; i < n; i++)
    for (int k = ai[i] - base; k < ai[i + 1] - base; k++) {
      const int c = aj[k] - base;
      if (uplo == LA_LOWER ? c >= i : c <= i) {
        set_error("la_trsv_analysis: row %d holds column %d outside the strict "
                  "%s triangle", i, c, uplo == LA_LOWER ? "lower" : "upper");
        return LA_ERR_INVALID_ARG;
      }
    }
  return LA_OK;
}

static la_status trsv_analysis_impl(la_uplo uplo, int n, int base, const int *ai,
                                    const int *aj, const double *av,
                                    const double *diag, la_dtype dtype,
                                    const int *iperm, const int *prefix,
                                    int nlevels, la_trsv_plan_t *out) {
  LA_CHECK_ARG(out && ai && n >= 0, "arguments");
  LA_CHECK_ARG(uplo == LA_LOWER || uplo == LA_UPPER, "uplo");
  LA_CHECK_ARG(dtype == LA_F64 || dtype == LA_F32, "dtype");
  LA_TRY(check_strict_triangle(uplo, n, base, ai, aj));
  if (iperm) {
    LA_CHECK_ARG(prefix && nlevels >= 0 && prefix[0] == 0 && prefix[nlevels] == n,
                 "level prefix must start at 0 and end at n");
    for (int l = 0; l < nlevels; l++)
      LA_CHECK_ARG(prefix[l + 1] >= prefix[l], "level prefix must be non-decreasing");
    std::vector<char> seen(n, 0);
    for (int p = 0; p < n; p++) {
      const int i = iperm[p] - base;
      LA_CHECK_ARG(i >= 0 && i < n && !seen[i], "iperm must be a permutation");
      seen[i] = 1;
    }
  }
  LA_TRY(require_device());
  std::unique_ptr<la_trsv_plan_s> P(new la_trsv_plan_s());
  P->n = n;
  P->nnz = ai[n] - base;
  P->base = base;
  P->uplo = uplo;
  P->dtype = dtype;
  P->unit = diag == nullptr;
  LA_TRY(trsv_build(P.get(), ai, aj, av, diag, iperm, prefix, nlevels));
  *out = P.release();
  return LA_OK;
}

la_status la_trsv_analysis(la_uplo uplo, int n, int base, const int *ai,
                           const int *aj, const double *av,
                           const double *diag, la_dtype dtype,
                           la_trsv_plan_t *out) {
  return trsv_analysis_impl(uplo, n, base, ai, aj, av, diag, dtype, nullptr, nullptr,
                            0, out);
}

la_status la_trsv_analysis_levels(la_uplo uplo, int n, int base, const int *ai,
                                  const int *aj, const double *av,
                                  const double *diag, la_dtype dtype,
                                  const int *iperm, const int *prefix,
                                  int nlevels, la_trsv_plan_t *out) {
  LA_CHECK_ARG(iperm && prefix, "iperm / prefix are NULL");
  return trsv_analysis_impl(uplo, n, base, ai, aj, av, diag, dtype, iperm, prefix,
                            nlevels, out);
}

la_status la_trsv_analysis_transposed(la_uplo uplo, int n, int base, const int *ai,
                                      const int *aj, const double *av,
                                      const double *diag, la_dtype dtype,
                                      la_trsv_plan_t *out) {
  LA_CHECK_ARG(out && ai && n >= 0, "arguments");
  LA_CHECK_ARG(uplo == LA_LOWER || uplo == LA_UPPER, "uplo");
  std::string why;
  if (!valid_csr(n, n, base, ai, aj, &why)) {
    set_error("invalid CSR: %s", why.c_str());
    return LA_ERR_BAD_CSR;
  }
  const int nnz = ai[n] - base;
  std::vector<int> tai(n + 1), taj(std::max(nnz, 1));
  std::vector<double> tav(std::max(nnz, 1));
  transpose(n, n, base, ai, aj, av, tai.data(), taj.data(), tav.data());
  return trsv_analysis_impl(uplo == LA_LOWER ? LA_UPPER : LA_LOWER, n, base, tai.data(),
                            taj.data(), tav.data(), diag, dtype, nullptr, nullptr, 0, out);
}

la_status la_trsv_partition(la_uplo uplo, int n, int base, const int *ai, const int *aj,
                           int nparts, int *part, int *coords) {
  LA_CHECK_ARG(ai && part && n >= 0 && nparts >= 1, "arguments");
  LA_CHECK_ARG(uplo == LA_LOWER || uplo == LA_UPPER, "uplo");
  LA_TRY(check_strict_triangle(uplo, n, base, ai, aj));
  int used = 0;
  if (n > 0) {
    std::vector<int> iperm(n), prefix(n + 1), lvl(n);
    const int levels = topological_sort2(uplo, n, base, ai, aj, iperm.data(), prefix.data());
    for (int l = 0; l < levels; l++)
      for (int p = prefix[l]; p < prefix[l + 1]; p++)
        lvl[iperm[p] - base] = l;
    std::vector<int> xadj, adj;
    undirected_pattern(n, base, ai, aj, xadj, adj);
    used = monotone_partition(n, xadj.data(), adj.data(), ai, aj, base, lvl.data(), nparts,
                              part);
  }
  if (coords)
    *coords = used;
  return LA_OK;
}

la_status la_trsv_partition_device(la_uplo uplo, int n, int base, const int *ai,
                                   const int *aj, int nparts, int *part, int *coords) {
  LA_CHECK_ARG(ai && part && n >= 0 && nparts >= 1, "arguments");
  LA_CHECK_ARG(uplo == LA_LOWER || uplo == LA_UPPER, "uplo");
  LA_TRY(check_strict_triangle(uplo, n, base, ai, aj));
  LA_TRY(require_device());
  int used = 0;
  if (n > 0) {
    std::vector<int> iperm(n), prefix(n + 1), lvl(n);
    const int levels = topological_sort2(uplo, n, base, ai, aj, iperm.data(), prefix.data());
    for (int l = 0; l < levels; l++)
      for (int p = prefix[l]; p < prefix[l + 1]; p++)
        lvl[iperm[p] - base] = l;
    la_status st = LA_OK;
    used = monotone_partition_device(n, base, ai, aj, lvl.data(), nparts, part, &st);
    if (used < 0)
      return st;
  }
  if (coords)
    *coords = used;
  return LA_OK;
}

la_status la_trsv(la_trsv_plan_t plan, const void *b, void *x,
                  la_stream_t stream) {
  LA_CHECK_ARG(plan && ((b && x) || plan->n == 0), "arguments");
  LA_CHECK_ARG(b != x || plan->n == 0, "b and x must not alias");
  LA_TRY(trsv_launch(plan, b, x, S(stream)));
  return trsv_check(plan, S(stream));
}

la_status la_trsv_launch(la_trsv_plan_t plan, const void *b, void *x,
                         la_stream_t stream) {
  LA_CHECK_ARG(plan && ((b && x) || plan->n == 0), "arguments");
  LA_CHECK_ARG(b != x || plan->n == 0, "b and x must not alias");
  return trsv_launch(plan, b, x, S(stream));
}

la_status la_trsv_status(la_trsv_plan_t plan, la_stream_t stream) {
  LA_CHECK_ARG(plan, "plan is NULL");
  return trsv_check(plan, S(stream));
}

la_status la_trsv_host(la_trsv_plan_t plan, const double *b, double *x) {
  LA_CHECK_ARG(plan && b && x, "arguments");
  LA_CHECK_ARG(plan->dtype == LA_F64, "host form takes an FP64 plan");
  if (!plan->hb.p) {
    LA_TRY(plan->hb.alloc(sizeof(double) * std::max(plan->n, 1)));
    LA_TRY(plan->hx.alloc(sizeof(double) * std::max(plan->n, 1)));
  }
  LA_CUDA_TRY(cudaMemcpy(plan->hb.p, b, sizeof(double) * plan->n, cudaMemcpyHostToDevice));
  LA_TRY(trsv_launch(plan, plan->hb.p, plan->hx.p, nullptr));
  LA_TRY(trsv_check(plan, nullptr));
  LA_CUDA_TRY(cudaMemcpy(x, plan->hx.p, sizeof(double) * plan->n, cudaMemcpyDeviceToHost));
  return LA_OK;
}

la_status la_trsv_levels(la_trsv_plan_t plan, int *levels, int *iperm,
                         int *prefix) {
  LA_CHECK_ARG(plan && levels, "arguments");
  *levels = plan->levels;
  if (iperm)
    std::memcpy(iperm, plan->h_iperm.data(), sizeof(int) * plan->n);
  if (prefix)
    std::memcpy(prefix, plan->h_prefix.data(), sizeof(int) * (plan->levels + 1));
  return LA_OK;
}

la_status la_trsv_schedule(la_trsv_plan_t plan, int *schedule, int *parts) {
  LA_CHECK_ARG(plan && schedule && parts, "arguments");
  *schedule = plan->sched == 1 && plan->ring_mask != la::kTrsvNoRing ? 2 : plan->sched;
  *parts = plan->sched == 1 ? plan->nparts : 0;
  return LA_OK;
}

la_status la_trsv_variant(la_trsv_plan_t plan, int *slots, int *second_row) {
  LA_CHECK_ARG(plan && slots && second_row, "arguments");
  *slots = plan->kd;
  *second_row = plan->sched == 1 && plan->w2 ? 1 : 0;
  return LA_OK;
}

la_status la_trsv_plan_destroy(la_trsv_plan_t plan) {
  delete plan;
  return LA_OK;
}

// ------------------------------------------------------------------- PCG
la_status la_pcg_create(la_csr_t A, const int *u_ai, const int *u_aj,
                        const double *icc_av, la_pcg_mode mode,
                        la_pcg_t *out) {
  LA_CHECK_ARG(A && u_ai && u_aj && icc_av && out, "arguments");
  LA_CHECK_ARG(A->n == A->ncols, "A must be square");
  LA_CHECK_ARG(A->dtype == LA_F64, "A must hold FP64 values");
  LA_CHECK_ARG(mode == LA_PCG_FP64 || mode == LA_PCG_MIXED, "mode");
  return pcg_create(A, u_ai, u_aj, icc_av, mode, out);
}

la_status la_pcg_solve(la_pcg_t s, const double *b, double *x, double rtol,
                       int maxit, la_pcg_info *info, la_stream_t stream) {
  LA_CHECK_ARG(s && b && x && b != x && rtol > 0 && maxit > 0, "arguments");
  return pcg_solve(s, b, x, rtol, maxit, info, S(stream));
}

la_status la_pcg_solve_host(la_pcg_t s, const double *b, double *x,
                            double rtol, int maxit, la_pcg_info *info) {
  LA_CHECK_ARG(s && b && x, "arguments");
  if (!s->hb.p) {
    LA_TRY(s->hb.alloc(sizeof(double) * std::max(s->n, 1)));
    LA_TRY(s->hx.alloc(sizeof(double) * std::max(s->n, 1)));
  }
  LA_CUDA_TRY(cudaMemcpy(s->hb.p, b, sizeof(double) * s->n, cudaMemcpyHostToDevice));
  const la_status st = pcg_solve(s, s->hb.as<double>(), s->hx.as<double>(),
                                 rtol, maxit, info, nullptr);
  LA_CUDA_TRY(cudaMemcpy(x, s->hx.p, sizeof(double) * s->n, cudaMemcpyDeviceToHost));
  return st;
}

la_status la_pcg_adjoint(la_pcg_t s, const double *g, const double *u,
                         double *dl_db, double *dl_dvalues, double rtol, int maxit,
                         la_pcg_info *info, la_stream_t stream) {
  LA_CHECK_ARG(s && g && u && dl_db && g != dl_db && rtol > 0 && maxit > 0, "arguments");
  return pcg_adjoint(s, g, u, dl_db, dl_dvalues, rtol, maxit, info, S(stream));
}

la_status la_pcg_fused(la_pcg_t s, int *fused) {
  LA_CHECK_ARG(s && fused, "arguments");
  *fused = s->fused ? 1 : 0;
  return LA_OK;
}

la_status la_pcg_destroy(la_pcg_t s) {
  pcg_destroy(s);
  return LA_OK;
}

} // extern "C"
