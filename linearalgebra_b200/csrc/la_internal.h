// la_internal.h -- shared internals of the B200 sparse hot path library.
#pragma once

#include "../../include/la_b200.h"

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

namespace la {

// ring_mask of a partitioned triangular-solve plan whose rows each have
// their own shared-memory slot
constexpr int kTrsvNoRing = 0x7fffffff;

// Thread-local last error message (la_last_error_string).
void set_error(const char *fmt, ...);
const char *get_error();

#define LA_CUDA_TRY(expr)                                                      \
  do {                                                                         \
    cudaError_t _e = (expr);                                                   \
    if (_e != cudaSuccess) {                                                   \
      ::la::set_error("%s failed: %s (%s:%d)", #expr, cudaGetErrorString(_e),  \
                      __FILE__, __LINE__);                                     \
      return LA_ERR_CUDA;                                                      \
    }                                                                          \
  } while (0)

#define LA_TRY(expr)                                                           \
  do {                                                                         \
    la_status _s = (expr);                                                     \
    if (_s != LA_OK)                                                           \
      return _s;                                                               \
  } while (0)

#define LA_CHECK_ARG(cond, msg)                                                \
  do {                                                                         \
    if (!(cond)) {                                                             \
      ::la::set_error("invalid argument: %s", msg);                            \
      return LA_ERR_INVALID_ARG;                                               \
    }                                                                          \
  } while (0)


// Returns LA_OK if a CUDA device of compute capability 10.x is current.
la_status require_device();
int sm_count();

// Device buffer with RAII release.
struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  ~DevBuf() { release(); }
  la_status alloc(size_t b);
  la_status upload(const void *host, size_t b);
  void release();
  template <typename T> T *as() const { return static_cast<T *>(p); }
};

// Ingest (la_ingest.cu): host readers of the reference's binary COO and of
// Matrix Market text, and the device build of a CSR from COO entries.
la_status read_file(const char *path, std::string &buf);
la_status read_binary_coo(const char *path, int base, std::vector<int> &rows,
                          std::vector<int> &cols, std::vector<double> &vals, int *m, int *n);
la_status parse_matrix_market(const char *text, size_t len, std::vector<int> &rows,
                              std::vector<int> &cols, std::vector<double> &vals, int *m,
                              int *n);
la_status csr_from_coo(int nrows, int ncols, long long nnz, int base, const int *rows,
                       const int *cols, const void *vals, la_dtype dtype, int flags,
                       la_csr_t *out);
// Device IC(0) / ILU(0) (la_factor.cu): kind 0 = IC(0) on the upper
// triangle with diagonals first, 1 = ILU(0) on a full pattern.
la_status factor_plan_create(int kind, int n, int base, const int *ai, const int *aj,
                             la_factor_plan_t *out);
la_status factor_numeric(la_factor_plan_t P, const double *av, double omega, double *out,
                         bool on_device, int *bad_row, cudaStream_t st);
// Stable LSD radix sort by (hi, lo) keys on the device (la_ingest.cu); the
// buffers [*cur] hold the input, *cur names the result's on return.
la_status radix_sort_pairs(int n, unsigned hi_range, unsigned lo_range, DevBuf (&kh)[2],
                           DevBuf (&kl)[2], DevBuf (&kp)[2], int *cur, cudaStream_t st);
// out[q] = base + (sorted keys below q) for q in [0, nq].
la_status run_starts(int n, const unsigned *sorted, int nq, int base, int *out, cudaStream_t st);
// TopologicalSort2 on the device (la_levels.cu), same outputs as
// topological_sort2; the triangle must be strict.
la_status topological_sort2_device(int uplo, int n, int base, const int *ai, const int *aj,
                                   int *iperm, int *prefix, int *levels);
// The same on a triangle already on the device (d_ai/d_aj carry base):
// order = rows sorted by (level, row), 0-based; keys = their levels; starts =
// the levels' first positions, levels + 1 entries.  Buffers are allocated.
la_status levels_on_device(int uplo, int n, int base, const int *d_ai, const int *d_aj,
                           DevBuf &order, DevBuf &keys, DevBuf &starts, int *levels,
                           cudaStream_t st);
// In-place exclusive prefix sum of d[0, m) on the device (la_ingest.cu).
la_status scan_exclusive(int *d, int m, cudaStream_t st);
// The optional FP32 copy of an FP64 matrix's values (LA_CSR_KEEP_F32).
la_status csr_finish(la_csr_t A, int flags);

// ------------------------------------------------------------ host algos
// (la_host.cpp) -- restatements of the reference's host-side steps.
bool valid_csr(int rows, int cols, int base, const int *ai, const int *aj,
               std::string *why);
int topological_sort2(int uplo, int n, int base, const int *ai, const int *aj,
                      int *iperm, int *prefix);
int topological_sort_kahn(int uplo, int n, int base, const int *ai, const int *aj, int *iperm,
                          int *prefix);
int ilu0(int n, int base, const int *ai, const int *aj, const double *av, double *lu);
void permute_vec(int n, int base, const double *v, const int *iperm, double *out);
void inverse_permute(int n, int base, const int *perm, int *iperm);
bool diagonal(int n, int base, const int *ai, const int *aj, const double *av, int *diagpos,
              double *diag, bool invert);
void transpose(int rows, int cols, int base, const int *ai, const int *aj,
               const double *av, int *t_ai, int *t_aj, double *t_av);
void permute(int n, int base, const int *ai, const int *aj, const double *av,
             const int *iperm, const int *perm, int *p_ai, int *p_aj,
             double *p_av);
void split_ldu(int n, int base, const int *ai, const int *aj, const double *av,
               int *l_ai, int *l_aj, double *l_av, double *d, int *u_ai,
               int *u_aj, double *u_av, int *lnnz, int *unnz);
int split_triangle(int uplo, int n, int base, const int *ai, const int *aj,
                   const double *av, int *t_ai, int *t_aj, double *t_av);
bool icc0(int n, int base, const int *u_ai, const int *u_aj, const double *u_av,
          double omega, double *icc_av);
// RCM (SerialCM); with `device` large components are ordered on the GPU.
constexpr int kRcmDeviceMin = 65536;
constexpr int kRcmMaxDegree = 64;
struct RcmDevice;
RcmDevice *rcm_device_create(int n, int base, const int *ai, const int *aj, const int *deg,
                             la_status *st);
void rcm_device_destroy(RcmDevice *D);
la_status rcm_device_component(RcmDevice *D, const int *members, int size, int *out);
la_status rcm_device_connected(int n, int base, const int *ai, const int *aj, int *iperm,
                               int *perm, bool *handled);
la_status rcm(int n, int base, const int *ai, const int *aj, int *iperm, int *perm,
              bool device = false);
// Row partition for the partitioned triangular solve (la_partition.cpp):
// k-d cuts on coordinates monotone along the dependency edges (row i reads
// row j for every stored (i, j) of dep_ptr/dep_col, which carry `base`), so
// the parts' dependency graph is acyclic.  xadj/adj: the 0-based undirected
// graph; lvl: the rows' levels.  Returns the number of coordinates used.
int monotone_partition(int n, const int *xadj, const int *adj, const int *dep_ptr,
                       const int *dep_col, int base, const int *lvl, int nparts, int *part);
// The same partition with its landmark stage on the GPU (graph, searches,
// candidate checks; LandmarksDevice below): identical parts.  Returns the
// coordinates used, or -1 with *st set when a device step failed.
int monotone_partition_device(int n, int base, const int *ai, const int *aj, const int *lvl,
                              int nparts, int *part, la_status *st);
// A candidate cut coordinate: sign * (d_a - d_b) for landmarks a < b (a = -1:
// the level), with its range over the vertices.
struct PartitionCand {
  int a, b, sign;
  long long range;
};
struct LandmarksDevice;
LandmarksDevice *landmarks_device_create(int n, int base, const int *ai, const int *aj,
                                         la_status *st);
la_status landmarks_device_candidates(LandmarksDevice *M, std::vector<PartitionCand> &cands);
la_status landmarks_device_coordinate(LandmarksDevice *M, const PartitionCand &c, int *f);
void landmarks_device_destroy(LandmarksDevice *M);

// The triangle's pattern made undirected and 0-based (both directions of
// every stored entry), the graph monotone_partition walks.
void undirected_pattern(int n, int base, const int *ai, const int *aj, std::vector<int> &xadj,
                        std::vector<int> &adj);

} // namespace la

// ----------------------------------------------------------------- handles
struct la_csr_s {
  int n = 0, ncols = 0, nnz = 0, base = 0;
  la_dtype dtype = LA_F64;
  la::DevBuf ai, aj, av, av32; // av32: FP32 copy of FP64 values (optional)
  std::vector<int> h_ai;       // host copy of the row pointers (plans)
  const void *values(la_dtype vd) const;
};

struct la_spmv_plan_s {
  la_csr_t A = nullptr;
  la_spmv_kind kind = LA_SPMV_SEGSUM;
  int ntiles = 0;
  la::DevBuf tile_row; // int[ntiles + 1]: row holding each tile's first nz
  la::DevBuf part;     // double[2 * ntiles]: head / tail partial sums
  la::DevBuf group_end; // int[ntiles]: end of the merge group a tile starts, else -1
  bool long_rows = true; // some row is longer than the per-thread row sum limit
  bool vec_tiles = false; // every row is short enough for the 16-byte load layout
  // row-slot form (rows of at most 8 entries): ell_k slots per row, slot-major
  // columns (-1 past a row's end) and values, FP64 and (if the matrix keeps
  // them) FP32; ell_k == 0: not used
  int ell_k = 0;
  la::DevBuf ell_j, ell_v, ell_v32;
  // lazily built transpose for the adjoint
  la_csr_t At = nullptr;
  la_spmv_plan_t Atplan = nullptr;
  std::vector<int> h_tile_row, h_group_end; // host copies (chunked host-pointer calls)
  // host staging for la_spmv_host: device copies of x and y, a stream for the
  // tile chunks, one for copying finished rows out, an event per chunk
  la::DevBuf hx, hy;
  cudaStream_t hst = nullptr, hcp = nullptr;
  cudaEvent_t hev[8] = {};
  ~la_spmv_plan_s() {
    for (cudaEvent_t e : hev)
      if (e)
        cudaEventDestroy(e);
    if (hst)
      cudaStreamDestroy(hst);
    if (hcp)
      cudaStreamDestroy(hcp);
  }
};

struct la_trsv_plan_s {
  int n = 0, nnz = 0, levels = 0, base = 0;
  la_uplo uplo = LA_LOWER;
  la_dtype dtype = LA_F64;
  bool unit = true;
  std::vector<int> h_iperm, h_prefix;
  // execution-ordered strict triangle: row p of the plan is original row
  // exec_row[p]; columns keep the original numbering.
  la::DevBuf ai, aj, av, diag, exec_row, chunk_start, err, ticket;
  int nchunks = 0;
  int grid = 0;
  int kd = 0; // dependency slots of the kernel variant (0: grouped form)
  int sleep_ns = 0; // level order: pause between polls of unpublished values
  // schedule: 0 = level order over the whole GPU with per-row readiness;
  // 1 = partitioned (one co-resident CTA per part, part values in shared
  // memory).  For schedule 1 the execution order is part-major, level-minor
  // and aj holds -1 - (position in the part) for a column of the same part.
  int sched = 0, nparts = 0, part_rows = 0;
  size_t part_smem = 0; // x slots of the largest part + its level boundaries
  int ring_mask = la::kTrsvNoRing; // x slots form a ring of ring_mask + 1 rows
  bool w2 = false; // partitioned kernel with the second-row register sets
  la::DevBuf pstart, psub, sb;
  la::DevBuf ej, ev; // first slots of every row, slot-major (schedule 1)
  // schedule 1 with 3-slot rows: per execution position {row, 3 columns}
  // (int4) and {3 values, diagonal} in the solve's type, instead of ej / ev
  la::DevBuf rmeta, rval;
  la::DevBuf hb, hx; // staging for the host form
};

struct la_pcg_s {
  la_csr_t A = nullptr;
  la_pcg_mode mode = LA_PCG_FP64;
  int n = 0;
  la_spmv_plan_t Ap = nullptr;
  la_trsv_plan_t L = nullptr, U = nullptr;
  la::DevBuf r, z, p, q, t;        // FP64 work vectors
  la::DevBuf r32, z32, p32, q32, t32, d32, p32b; // FP32 inner vectors (mixed)
  la::DevBuf scal, partials, ticket;
  la::DevBuf bar; // grid barrier of the fused kernels: arrivals, generation, error
  la::DevBuf hb, hx;
  int dot_blocks = 0;
  // the iteration's vector work in two cooperative kernels (dot products
  // finished inside them) instead of separate dot / update launches
  bool fused = true;
  // mixed mode: the reliable update falls due when the FP32 residual has
  // dropped by this factor; the next step is queued ahead of the residual's
  // arrival while the last residual is above ahead_margin times that
  double reliable_delta = 0.1, ahead_margin = 1.3;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double *h_rr = nullptr;       // pinned host copy of the residual norm
  cudaEvent_t ev_rr = nullptr;  // marks its arrival
};

// Device IC(0) / ILU(0) plan (la_factor.cu).
struct la_factor_plan_s {
  int kind = 0; // 0: IC(0), 1: ILU(0)
  int n = 0, nnz = 0, base = 0, levels = 0, nchunks = 0, grid = 0;
  int sleep_ns = 0; // the numeric pass's pause between polls of unpublished rows
  long long npairs = 0; // (target, source) pairs of all updates
  bool warp = false;    // numeric pass: one warp per row (many pairs a row)
  // per row (original numbering): its value range [rs, re) and its diagonal
  la::DevBuf rs, diag;
  // rows in execution order, 32-row chunks that never cross a level
  la::DevBuf exec_row, chunk_start;
  // per row: its updates [uptr[j], uptr[j+1]); per update: source row k,
  // scalar index (IC: U_kj in row k; ILU: the row's own L_jk entry), pivot
  // index (ILU: row k's diagonal), and its pairs [pptr[u], pptr[u+1])
  la::DevBuf uptr, uk, us, upiv, pptr, ptgt, psrc;
  la::DevBuf vin, done, state; // state: ticket, timeout flag, smallest bad row
  std::vector<int> h_ai;
};
