/* la_b200.h -- C-ABI of the B200-native sparse hot path.
 *
 * Drop-in replacement, for one NVIDIA B200 (sm_100a), of the sparse hot
 * path of miaodi/linearAlgebra: CSR SpMV in its segmented-sum and ALBUS
 * forms, the level-scheduled triangular solves that apply IC(0)/ILU(0)
 * factors, the IC(0)-preconditioned CG built on them, and hand-written
 * adjoints.  Every entry point below names the reference interface it
 * replaces (path:line within the reference project).
 *
 * Conventions (those of the reference, sparse_mat_op/spmv.hpp:16-19):
 *  - CSR with int32 row pointers `ai[n+1]` and column indices `aj[nnz]`,
 *    index base 0 or 1 (ai[0] == base), values double (LA_F64) or float
 *    (LA_F32);
 *  - SpMV computes y = alpha * A * x + beta * y (the reference names the
 *    input b and the output x); when beta == 0, y is not read;
 *  - the caller owns every array passed in; handles own device copies;
 *  - a handle is used from one stream and one host thread at a time, as the
 *    reference objects are (their operator() mutates scratch);
 *  - pointers passed to the `_host` entry points are host memory; all other
 *    vector pointers are device memory;
 *  - every call returns an la_status; la_last_error_string() describes the
 *    last failure of the calling thread.
 * No function here falls back to the CPU: without a usable CUDA device the
 * device entry points return LA_ERR_NO_DEVICE.
 */
#ifndef LA_B200_H
#define LA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  LA_OK = 0,
  LA_ERR_INVALID_ARG = 1,
  LA_ERR_BAD_CSR = 2,       /* fails ValidCSR (matrix_utils.hpp:985-1014) */
  LA_ERR_CUDA = 3,          /* a CUDA runtime call failed */
  LA_ERR_TIMEOUT = 4,       /* a bounded device wait gave up */
  LA_ERR_BREAKDOWN = 5,     /* IC pivot < 0 (precond.hpp:684-685) */
  LA_ERR_NOT_CONVERGED = 6, /* iteration limit reached */
  LA_ERR_NO_DEVICE = 7,     /* no usable sm_100 device */
  LA_ERR_ALLOC = 8
} la_status;

typedef enum { LA_F64 = 0, LA_F32 = 1 } la_dtype;

typedef enum {
  LA_SPMV_SEGSUM = 0, /* SegSumSPMV, sparse_mat_op/spmv.hpp:59-185 */
  LA_SPMV_ALBUS = 1   /* ALBUSSPMV,  sparse_mat_op/spmv.hpp:186-300 */
} la_spmv_kind;

typedef enum { LA_LOWER = 0, LA_UPPER = 1 } la_uplo; /* TriangularMatrix L/U,
                                                        matrix_utils.hpp:581 */

typedef struct la_csr_s *la_csr_t;
typedef struct la_spmv_plan_s *la_spmv_plan_t;
typedef struct la_trsv_plan_s *la_trsv_plan_t;
typedef struct la_pcg_s *la_pcg_t;
typedef struct la_factor_plan_s *la_factor_plan_t;
typedef void *la_stream_t; /* a cudaStream_t; NULL is the legacy stream */

/* ---------------------------------------------------------------- misc */
const char *la_last_error_string(void);
/* Library version string. */
const char *la_version(void);
/* Number of SMs of the current device (0 if none); a liveness probe. */
la_status la_device_sm_count(int *sms);

/* ---------------------------------------------------------- CSR handle */
/* Device copy of a CSR matrix (the reference's CSRMatrix* containers,
 * matrix_utils.hpp:37-103).  ai/aj/av are HOST arrays; the structure is
 * validated with ValidCSR semantics (matrix_utils.hpp:985-1014: ai[0] ==
 * base, rows sorted, no duplicates, columns in range) before upload.
 * `flags` bit 0 (LA_CSR_KEEP_F32): also keep an FP32 copy of FP64 values,
 * used by the mixed-precision solver. */
#define LA_CSR_KEEP_F32 1
la_status la_csr_create(int n, int ncols, int base, const int *ai,
                        const int *aj, const void *av, la_dtype dtype,
                        int flags, la_csr_t *out);
/* Same, from DEVICE arrays (copied; no validation beyond sizes). */
la_status la_csr_create_device(int n, int ncols, int nnz, int base,
                               const int *d_ai, const int *d_aj,
                               const void *d_av, la_dtype dtype, int flags,
                               la_csr_t *out);
/* Replace the values (same pattern); av is host memory if on_device == 0. */
la_status la_csr_update_values(la_csr_t A, const void *av, int on_device);
la_status la_csr_info(la_csr_t A, int *n, int *ncols, int *nnz, int *base,
                      la_dtype *dtype);
la_status la_csr_destroy(la_csr_t A);
/* Host copies of a handle's arrays (ai[n+1], aj[nnz], av[nnz] in its dtype);
 * any pointer may be NULL to skip that array. */
la_status la_csr_download(la_csr_t A, int *ai, int *aj, void *av);

/* ---------------------------------------------------------------- ingest */
/* The on-disk formats either side of the path (utils/utils.h:23-132).
 *
 * la_csr_from_coo: a device CSR from HOST coordinate entries (indices carry
 * `base`: rows[k] - base in [0, nrows), cols[k] - base in [0, ncols)),
 * ordered by (row, col) on the device -- the construction ReadFromBinaryCSR
 * (utils.h:46-91) and read_matrix_market_csr (utils.h:93-132) perform on the
 * host.  Entries with equal (row, col) are kept, in input order. */
la_status la_csr_from_coo(int nrows, int ncols, long long nnz, int base, const int *rows,
                          const int *cols, const void *vals, la_dtype dtype, int flags,
                          la_csr_t *out);
/* ReadFromBinaryCOO (utils.h:23-44), host only: the file is an int64 entry
 * count followed by std::tuple<int32 row, int32 col, double value> records
 * (16 bytes each as libstdc++ lays the tuple out: value, col, row); *m /
 * *n = largest row / column index + 1 - base, as the reference returns them.
 * Call with rows == cols == vals == NULL to learn *nnz, then again with
 * arrays of *nnz entries (entries in file order). */
la_status la_read_binary_coo(const char *path, int base, long long *nnz, int *rows, int *cols,
                             double *vals, int *m, int *n);
/* A Matrix Market coordinate file (real, integer or pattern; general,
 * symmetric or skew-symmetric), host only, as 0-based entries: symmetric
 * storage expanded by mirroring every off-diagonal entry (the reference reads
 * through fast_matrix_market with its symmetry generalisation), pattern
 * entries valued 1.  Two-call pattern as above. */
la_status la_read_matrix_market(const char *path, long long *nnz, int *rows, int *cols,
                                double *vals, int *m, int *n);
/* ReadFromBinaryCSR (utils.h:46-91) into a device CSR with the file's base,
 * and read_matrix_market_csr (utils.h:93-132) into a 0-based device CSR
 * (from a file, or from the text already in memory). */
la_status la_csr_read_binary_coo(const char *path, int base, int flags, la_csr_t *out);
la_status la_csr_read_matrix_market(const char *path, int flags, la_csr_t *out);
la_status la_csr_parse_matrix_market(const char *text, size_t len, int flags, la_csr_t *out);

/* ---------------------------------------------------------------- SpMV */
/* Plan = the reference's preprocess() (SegSumSPMV::preprocess,
 * spmv.hpp:68-77; ALBUSSPMV::preprocess, spmv.hpp:195-228): the nnz are cut
 * into equal tiles and the start row of every tile is found by binary
 * search, once.  Scratch for cross-tile partial rows is owned by the plan. */
la_status la_spmv_plan_create(la_csr_t A, la_spmv_kind kind,
                              la_spmv_plan_t *out);
/* y = alpha*A*x + beta*y on the device (SegSumSPMV::operator(),
 * spmv.hpp:79-177; ALBUSSPMV::operator(), spmv.hpp:230-293; SPMV<>
 * adapter, spmv.hpp:326-330).  x, y device arrays of `vdtype`: LA_F64 needs
 * an FP64 matrix; LA_F32 vectors use the FP32 values (an FP32 matrix or the
 * LA_CSR_KEEP_F32 copy) and accumulate in FP32. */
la_status la_spmv(la_spmv_plan_t plan, double alpha, const void *x,
                  double beta, void *y, la_dtype vdtype, la_stream_t stream);
/* Host-pointer form of the same call: x (n doubles) is copied in, y copied
 * in when beta != 0 and out always; synchronous.  This is the path the
 * C++ drop-in classes (include/la_b200.hpp) take for host vectors. */
la_status la_spmv_host(la_spmv_plan_t plan, double alpha, const double *x,
                       double beta, double *y);
la_status la_spmv_plan_destroy(la_spmv_plan_t plan);
/* The layout the plan's SpMV runs on (no reference counterpart):
 * *row_slots = 0 for the nnz-balanced tile pass (1024-nonzero tiles, rows
 * crossing a tile combined from partial sums in the reference's merge
 * order), or k > 0 for the row-slot form the plan picks for matrices of at
 * least 65,536 rows whose rows all hold at most 8 entries (k slots a row,
 * padding at most a quarter): every row then summed by one thread in stored
 * order, SerialSPMV's row sum formed as SegSum / ALBUS form it. */
la_status la_spmv_layout(la_spmv_plan_t plan, int *row_slots);
/* Measurement aid (no reference counterpart; not an SpMV): the bound a
 * matrix sets for the SpMV tile pass.  One launch streams the plan's FP64
 * matrix (columns and values, 16-byte loads, whole 1024-nonzero tiles) and,
 * when gather != 0, also gathers the device vector x through the columns --
 * the tile pass without its row structure.  sink: one device double that is
 * never written in practice.  Time it like la_spmv; its algorithmic bytes
 * are nnz * 12 (whole tiles). */
la_status la_spmv_ceiling(la_spmv_plan_t plan, const double *x, int gather, double *sink,
                          la_stream_t stream);

/* Allocation-free SpMV.  No counterpart in the reference (which has no
 * device code); it exists for callers that must not allocate device memory:
 * code embedded in an application that hands out the whole device memory
 * budget through its own pool, where a library cudaMalloc would fail or
 * break that budget, and latency-critical loops that cannot take the
 * implicit device-wide synchronisation of cudaMalloc / cudaFree.
 * y = alpha*A*x + beta*y in FP64 with the SegSum or ALBUS form, from DEVICE
 * CSR arrays (d_ai[n+1], d_aj[nnz], d_av[nnz], base 0 or 1), d_x (ncols
 * entries) and d_y (n entries, not aliasing d_x); the result equals
 * la_spmv's.  The arrays are used as given, without the host validation
 * la_csr_create does: d_ai[0] must equal base and d_ai[n] - base must equal
 * nnz.  If not, the result is undefined, but no write leaves d_y[0, n) and
 * no read of d_aj / d_av goes beyond the nnz entries declared.  No
 * cudaMalloc, cudaFree or allocating library call is made:
 * the scratch lives in a fixed device array of 655,616 bytes that every GPU
 * loading the library holds until the process exits, so nnz is limited to
 * LA_SPMV_NOALLOC_MAX_NNZ (larger inputs return LA_ERR_INVALID_ARG).  The
 * first call on a device looks up that array's device address (a one-time
 * set-up per device); make that first call before any stream capture.  All
 * calls share the array: each call rewrites what it reads, so nothing has
 * to start at zero, but calls whose kernels overlap on the GPU (other
 * streams, other host threads) race on it. */
#define LA_SPMV_NOALLOC_MAX_NNZ (32768 * 1024)
la_status la_spmv_noalloc(la_spmv_kind kind, int n, int nnz, int base,
                          const int *d_ai, const int *d_aj, const double *d_av,
                          double alpha, const double *d_x, double beta,
                          double *d_y, la_stream_t stream);

/* Row-block SpMV of a distributed matrix (no reference counterpart; the
 * reference's ParallelSPMV splits rows over threads by equal nonzero shares,
 * utils/utils.h:187-222, which is how the blocks are cut across GPUs).  The
 * plan's matrix is this rank's block of rows with global column indices;
 * x is not gathered into one array first: it stays split into `nparts`
 * contiguous slices, slice r holding columns [part_start[r],
 * part_start[r+1]) at xparts[r], a device pointer that may be another GPU's
 * memory mapped into this one (peer access or symmetric memory), and the
 * kernel reads every column from the slice that owns it.  part_start is a
 * HOST array of nparts + 1 non-decreasing entries from 0 to the matrix's
 * column count; 1 <= nparts <= LA_SPMV_MAX_XPARTS.  The values of x must be
 * in place before the call (the caller orders the writers, e.g. by a
 * barrier across ranks); y = alpha*A*x + beta*y in the dtype of the slices. */
#define LA_SPMV_MAX_XPARTS 8
la_status la_spmv_xparts(la_spmv_plan_t plan, double alpha, const void *const *xparts,
                         const int *part_start, int nparts, double beta, void *y,
                         la_dtype vector_dtype, la_stream_t stream);

/* Adjoints of y = A x (no reference counterpart; the reference has none).
 * la_spmv_transpose: out = alpha * A^T g + beta * out (dL/dx), through a
 * transposed copy of A built once per plan on first use (the role
 * ForwardSubstitutionT plays for triangles, triangle_solve.hpp:87-98).
 * la_sddmm_pattern: dv[k] = alpha * g[row(k)] * x[col(k)] over the stored
 * pattern (dL/dvalues).  FP64 only. */
la_status la_spmv_transpose(la_spmv_plan_t plan, double alpha, const double *g,
                            double beta, double *out, la_stream_t stream);
la_status la_sddmm_pattern(la_spmv_plan_t plan, double alpha, const double *g,
                           const double *x, double *dv, la_stream_t stream);

/* ------------------------------------------------------- host analysis */
/* TopologicalSort<L|U> (matrix_utils.hpp:583-635, Kahn's breadth-first
 * order), bit-identical output: the same level sets as TopologicalSort2,
 * rows of a level in breadth-first order (level 0 ascending for L,
 * descending for U; then the readers of each row as its level is walked).
 * *result is the reference's return value -- the index of the last level
 * (levels - 1; 0 for n == 0) -- and prefix receives *result + 2 zero-based
 * entries (caller provides n + 2 ints); iperm values carry the base.
 * LA_ERR_INVALID_ARG if the entries form a cycle (the reference loops). */
la_status la_topological_sort(la_uplo uplo, int n, int base, const int *ai, const int *aj,
                              int *iperm, int *prefix, int *result);
/* TopologicalSort2<L|U> (matrix_utils.hpp:637-675), bit-identical output:
 * iperm[n] (values i + base, ordered by level then row) and zero-based
 * prefix[levels + 1] (caller provides n + 1 ints).  Returns the level
 * count in *levels. */
la_status la_topological_sort2(la_uplo uplo, int n, int base, const int *ai,
                               const int *aj, int *iperm, int *prefix,
                               int *levels);
/* The same level sets computed on the GPU (no reference counterpart beyond
 * TopologicalSort2 itself): the depths as a (max, +) triangular solve in one
 * persistent launch, the rows ordered by a stable radix sort on their depth.
 * Host arrays in and out, outputs identical to la_topological_sort2.  The
 * triangle must be strict (LA_ERR_INVALID_ARG otherwise).  The triangular
 * solve analysis uses it for triangles of at least 65,536 rows. */
la_status la_topological_sort2_device(la_uplo uplo, int n, int base, const int *ai,
                                      const int *aj, int *iperm, int *prefix, int *levels);
/* SerialCM reverse Cuthill-McKee (reordering/Reordering.cpp:37-136),
 * bit-identical iperm/perm (values carry the base). */
la_status la_rcm(int n, int base, const int *ai, const int *aj, int *iperm,
                 int *perm);
/* The same ordering with its large components ordered on the GPU (no
 * reference counterpart beyond SerialCM itself): components of at least
 * 65,536 nodes, when no row holds more than 64 entries, get their
 * pseudo-peripheral search as level-synchronous device BFS and their
 * Cuthill-McKee sweep as per-level device steps (parents, child counts, a
 * scan, per-parent sorts by (degree, index)); the rest as la_rcm.  The
 * outputs are identical to la_rcm's. */
la_status la_rcm_device(int n, int base, const int *ai, const int *aj, int *iperm,
                        int *perm);
/* ILU(0) on A's own pattern, from scratch (no reference counterpart: the
 * reference factors ILU through MKL, and its level-0 path never fills the
 * upper-part positions, incomplete_lu.cpp:166 / :267-269).  lu_av (A's
 * pattern) receives L strictly below the diagonal (unit diagonal implied)
 * and U on and above it, so that (L U)_ij = A_ij on the pattern; split it
 * with la_split_ldu and apply it with a unit-lower and an upper la_trsv plan,
 * as incomplete_lu.cpp:36-48 does.  Rows' columns sorted, every diagonal
 * stored (LA_ERR_INVALID_ARG otherwise); LA_ERR_BREAKDOWN on a zero pivot. */
la_status la_ilu0(int n, int base, const int *ai, const int *aj, const double *av,
                  double *lu_av);
/* permuteVec (matrix_utils.hpp:562-576): out[i] = v[iperm[i] - base], or a
 * copy when iperm is NULL. */
la_status la_permute_vec(int n, int base, const double *v, const int *iperm, double *out);
/* inversePermute (utils/utils.cpp:101-108): iperm[perm[i] - base] = i + base;
 * LA_ERR_INVALID_ARG unless perm is a permutation. */
la_status la_inverse_permute(int n, int base, const int *perm, int *iperm);
/* Diagonal (matrix_utils.hpp:677-704): per row the position (with base) of
 * the diagonal entry in diagpos and its value in diag (either may be NULL;
 * with invert != 0, 1/value, 0 giving 1); *all_present = the reference's
 * bool (0 when some row has no diagonal entry: its position is then where
 * the entry would go and its value what is stored there, 0 past the last
 * entry, where the reference reads beyond its arrays).  Rows' columns must
 * be sorted (LA_ERR_BAD_CSR otherwise). */
la_status la_diagonal(int n, int base, const int *ai, const int *aj, const double *av,
                      int *diagpos, double *diag, int invert, int *all_present);
/* permute (matrix_utils.hpp:429-472): B(i,:) = A(iperm[i],:), columns mapped
 * through perm (may be NULL: rows only, permuteRow :474-480) and re-sorted. */
la_status la_permute(int n, int base, const int *ai, const int *aj,
                     const double *av, const int *iperm, const int *perm,
                     int *p_ai, int *p_aj, double *p_av);
/* ParallelTranspose2 (matrix_utils.hpp:311-390). av/t_av may be NULL. */
la_status la_transpose(int rows, int cols, int base, const int *ai,
                       const int *aj, const double *av, int *t_ai, int *t_aj,
                       double *t_av);
/* SplitLDU (matrix_utils.hpp:720-803); outputs sized nnz / n + 1 / n. */
la_status la_split_ldu(int n, int base, const int *ai, const int *aj,
                       const double *av, int *l_ai, int *l_aj, double *l_av,
                       double *d, int *u_ai, int *u_aj, double *u_av,
                       int *lnnz, int *unnz);
/* SplitTriangle<L|U> (matrix_utils.hpp:805-879), incl. the diagonal. */
la_status la_split_triangle(la_uplo uplo, int n, int base, const int *ai,
                            const int *aj, const double *av, int *t_ai,
                            int *t_aj, double *t_av, int *tnnz);
/* ValidCSR (matrix_utils.hpp:985-1014): LA_OK or LA_ERR_BAD_CSR. */
la_status la_valid_csr(int rows, int cols, int base, const int *ai,
                       const int *aj);
/* IC(0) numeric factor, ICCLevel0SymSymbolic + ICCLevelNumeric
 * (precond.hpp:13-37, 615-693): u_* is the upper triangle of an SPD matrix
 * with the diagonal first in each row; icc_av (same pattern) receives U
 * with A ~= U^T U.  omega shifts the diagonal by (1 + omega).
 * LA_ERR_BREAKDOWN on a negative pivot. */
la_status la_icc0(int n, int base, const int *u_ai, const int *u_aj,
                  const double *u_av, double omega, double *icc_av);
/* incomplete_cholesky_k_2::numeric_factorize shift-retry loop
 * (mkl_wrapper/incomplete_cholesky.cpp:315-342): on breakdown retry with
 * shift = max(2 * shift, 1e-3), at most 20 restarts.  *shift_used gets the
 * final shift. */
la_status la_icc0_shifted(int n, int base, const int *u_ai, const int *u_aj,
                          const double *u_av, double *icc_av,
                          double *shift_used);

/* The same factorisations on the GPU: a symbolic plan built once per
 * pattern (every row's updates in the order the sequential algorithm
 * applies them, found per row in parallel -- for IC(0) patterns of at least
 * 65,536 rows on the GPU, else on the host), then numeric passes on the
 * device, one persistent launch each, level-scheduled by the rows'
 * dependencies -- bit-identical to la_icc0 / la_ilu0 (same operations, same
 * order).  For a pattern factored more than once (new values, shift
 * retries) the numeric pass replaces the host's.
 * la_icc0_plan_create: u_ai/u_aj as la_icc0 takes them (ICCLevelNumeric,
 * precond.hpp:615-693), each row's columns strictly ascending from its
 * diagonal (LA_ERR_INVALID_ARG otherwise).  la_ilu0_plan_create: a full pattern, every row
 * holding its diagonal, as la_ilu0 takes it.  HOST arrays. */
la_status la_icc0_plan_create(int n, int base, const int *u_ai, const int *u_aj,
                              la_factor_plan_t *out);
la_status la_ilu0_plan_create(int n, int base, const int *ai, const int *aj,
                              la_factor_plan_t *out);
/* Numeric pass: values av in (the plan's pattern order), the factor out (same
 * pattern); both host arrays when on_device == 0, device arrays otherwise
 * (synchronises `stream`).  omega shifts IC(0)'s diagonal by (1 + omega)
 * (ignored for ILU(0)).  LA_ERR_BREAKDOWN on a negative IC(0) pivot or a zero
 * ILU(0) pivot, with *bad_row (if non-NULL) the smallest such row -- where
 * the sequential algorithm stops; -1 otherwise. */
la_status la_factor_numeric(la_factor_plan_t plan, const double *av, double omega,
                            double *out, int on_device, int *bad_row, la_stream_t stream);
/* la_icc0_shifted's retry loop (incomplete_cholesky.cpp:315-342) over device
 * numeric passes. */
la_status la_factor_icc0_shifted(la_factor_plan_t plan, const double *av, double *out,
                                 int on_device, double *shift_used, la_stream_t stream);
/* Number of dependency levels of the plan's rows. */
la_status la_factor_levels(la_factor_plan_t plan, int *levels);
la_status la_factor_plan_destroy(la_factor_plan_t plan);

/* ------------------------------------------------- triangular solves */
/* OptimizedTriangularSolve<Barrier, L|U>::analysis (triangle_solve.hpp:
 * 157-159, triangle_solve.tpp:17-113): levels by TopologicalSort2 on the
 * host, rows stored in execution (level) order, uploaded once.  ai/aj/av:
 * HOST CSR of the STRICT triangle; diag: host array of n values or NULL
 * (unit diagonal).  `dtype` selects FP64 or FP32 storage (FP32 values and
 * FP32 vectors in la_trsv).  One kernel launch per solve, with one of two
 * schedules chosen here by a cost model (see la_trsv_schedule): the level
 * order over the whole GPU with per-row readiness, or a partition of the
 * rows into co-resident CTAs that keep their rows' values in shared memory
 * and hand values across parts through global memory.  Every wait is
 * bounded. */
la_status la_trsv_analysis(la_uplo uplo, int n, int base, const int *ai,
                           const int *aj, const double *av,
                           const double *diag, la_dtype dtype,
                           la_trsv_plan_t *out);
/* Same, with a caller-built level structure instead of TopologicalSort2's:
 * iperm[n] (values carry the base) and zero-based prefix[nlevels + 1], the
 * form TopologicalSort2 returns (matrix_utils.hpp:637-675) and
 * LevelScheduleForward/BackwardSubstitution consume (triangle_solve.hpp:
 * 100-145).  iperm must be a permutation and prefix run from 0 to n; that
 * every row comes after the rows it reads is the caller's promise -- if it
 * is broken, a solve may stall, and its bounded waits then end it with
 * LA_ERR_TIMEOUT. */
la_status la_trsv_analysis_levels(la_uplo uplo, int n, int base,
                                  const int *ai, const int *aj,
                                  const double *av, const double *diag,
                                  la_dtype dtype, const int *iperm,
                                  const int *prefix, int nlevels,
                                  la_trsv_plan_t *out);
/* The transposed solve: a plan that solves with T^T, given the CSR of the
 * strict triangle T (`uplo` names T's triangle; the plan's is the other).
 * With diag = NULL and T strict upper this is ForwardSubstitutionT
 * (triangle_solve.hpp:87-98: the unit lower solve with L = U^T, which the
 * reference runs as a column scatter); with a diag, (T^T + D) x = b.  T^T
 * is formed on the host once (ParallelTranspose2 order, matrix_utils.hpp:
 * 311-390), then planned as la_trsv_analysis does.  The scatter subtracts
 * each product from x_j in turn while the plan sums a row first: FP64
 * results agree to rounding, not bit for bit. */
la_status la_trsv_analysis_transposed(la_uplo uplo, int n, int base, const int *ai,
                                      const int *aj, const double *av,
                                      const double *diag, la_dtype dtype,
                                      la_trsv_plan_t *out);
/* The row partition the partitioned schedule cuts for this strict triangle
 * (no reference counterpart; host only, needs no GPU): part[n] in
 * [0, nparts), from value cuts on coordinates monotone along the
 * dependencies, so that a row never reads a row of a higher-numbered part
 * (part[j] <= part[i] whenever row i reads row j); *coords (may be NULL)
 * receives the number of cut coordinates found (3 for a 7-point grid, 1 --
 * the level alone -- when no other is monotone).  The analysis uses this
 * partition with nparts = one per SM when its cost model prefers it. */
la_status la_trsv_partition(la_uplo uplo, int n, int base, const int *ai, const int *aj,
                            int nparts, int *part, int *coords);
/* The same partition with its landmark stage on the GPU -- the undirected
 * graph, the landmark searches and the candidate checks -- as the analysis
 * computes it; part and *coords identical to la_trsv_partition's.  HOST
 * arrays; needs a device (LA_ERR_NO_DEVICE otherwise). */
la_status la_trsv_partition_device(la_uplo uplo, int n, int base, const int *ai,
                                   const int *aj, int nparts, int *part, int *coords);
/* x = T^-1 b (triangle_solve.tpp:115-155 operator()/BarrierOp): b, x device
 * arrays of the plan's dtype; b and x must not alias.  LA_ERR_TIMEOUT if a
 * dependency wait exceeded its bound (x is then undefined). */
la_status la_trsv(la_trsv_plan_t plan, const void *b, void *x,
                  la_stream_t stream);
/* Asynchronous form of la_trsv: launches and returns without waiting; a
 * timeout is recorded in the plan and reported by la_trsv_status. */
la_status la_trsv_launch(la_trsv_plan_t plan, const void *b, void *x,
                         la_stream_t stream);
/* Synchronises `stream` and returns LA_ERR_TIMEOUT if any launch of this
 * plan since the last status check gave up on a wait (then clears it). */
la_status la_trsv_status(la_trsv_plan_t plan, la_stream_t stream);
/* Host-pointer form (synchronous). */
la_status la_trsv_host(la_trsv_plan_t plan, const double *b, double *x);
/* Level structure of the plan: *levels, and if non-NULL iperm[n] /
 * prefix[levels + 1] exactly as TopologicalSort2 returns them. */
la_status la_trsv_levels(la_trsv_plan_t plan, int *levels, int *iperm,
                         int *prefix);
/* Schedule the analysis chose (no reference counterpart; all compute the
 * same bits): *schedule = 0 for level order over the whole GPU with per-row
 * readiness, 1 for the partitioned form (*parts co-resident CTAs, each
 * keeping its rows' values in shared memory), 2 for the partitioned form
 * whose parts are too large for shared memory, which keeps each part's most
 * recent rows in a shared-memory ring and reads older ones from x.  Set
 * LA_TRSV_SCHEDULE=flags or =parts in the environment before the analysis to
 * force level order or a partition; LA_TRSV_RING=<rows> (a power of two, at
 * least 32) forces a ring of that size onto a partition. */
la_status la_trsv_schedule(la_trsv_plan_t plan, int *schedule, int *parts);
/* Kernel variant of the plan (no reference counterpart; every variant
 * computes the same bits): *slots = the number of leading entries of a row
 * held in registers (3, 4, 8 or 16; 0 for the grouped level-order form whose
 * rows are read in groups of 8), *second_row = 1 when the partitioned FP32
 * kernel holds each thread's second row of a level in registers too (chosen
 * when some level of a part is wider than the CTA; LA_TRSV_W2=0 in the
 * environment before the analysis keeps it off). */
la_status la_trsv_variant(la_trsv_plan_t plan, int *slots, int *second_row);
la_status la_trsv_plan_destroy(la_trsv_plan_t plan);

/* ---------------------------------------------------------- IC(0)-PCG */
/* Solver state for A x = b with the IC(0) preconditioner U^T U; the role of
 * mkl_pcg_solver + incomplete_cholesky_k_2 (mkl_wrapper/mkl_solver.cpp:
 * 150-251, mkl_wrapper/incomplete_cholesky.cpp:21-29, 286-342).
 * A: FP64 CSR handle (full symmetric storage).  u_ai/u_aj/icc_av: HOST IC
 * factor U (upper, diagonal first, as la_icc0 returns).  mode LA_PCG_FP64:
 * everything FP64.  mode LA_PCG_MIXED: FP64 iterative refinement by
 * reliable updates -- the CG recurrence runs on FP32 vectors whose SpMV and
 * triangular solves read FP32 A / FP32 factors and accumulate in FP32, with
 * FP64 dot products and scalars; whenever its residual has dropped tenfold,
 * x is updated in FP64 and the residual is replaced by r = b - A x computed
 * with the FP64 matrix, keeping the search direction. */
typedef enum { LA_PCG_FP64 = 0, LA_PCG_MIXED = 1 } la_pcg_mode;
typedef struct {
  int iterations;        /* total (inner) PCG iterations */
  int outer_iterations;  /* FP64 residual replacements (1 for FP64) */
  double rel_residual;   /* true ||b - A x|| / ||b|| in FP64 at exit */
  double solve_ms;       /* device time of the solve, CUDA events */
} la_pcg_info;
la_status la_pcg_create(la_csr_t A, const int *u_ai, const int *u_aj,
                        const double *icc_av, la_pcg_mode mode,
                        la_pcg_t *out);
/* Solve to ||b - A x|| / ||b|| < rtol (the reference's user stopping test,
 * mkl_solver.cpp:211-225), x0 = 0.  b, x: device FP64 arrays.
 * LA_ERR_NOT_CONVERGED if maxit is reached (x holds the last iterate). */
la_status la_pcg_solve(la_pcg_t s, const double *b, double *x, double rtol,
                       int maxit, la_pcg_info *info, la_stream_t stream);
/* Host-pointer form (synchronous): b, x host arrays of n doubles. */
la_status la_pcg_solve_host(la_pcg_t s, const double *b, double *x,
                            double rtol, int maxit, la_pcg_info *info);
/* Adjoint of u = A^-1 b through a full solve (no reference counterpart; the
 * reference has no derivatives).  For a loss L(u) with g = dL/du (device):
 * lambda = A^-T g by one more preconditioned CG solve with the same operator
 * (A is symmetric), returned as dl_db = dL/db; if dl_dvalues is non-NULL it
 * receives dL/dA over A's stored pattern, -lambda_i * u_j for entry (i, j)
 * (nnz values, A's order).  u is the forward solution (device).  For a
 * symmetric parameterisation (a_ij and a_ji one parameter) add the two
 * mirrored entries. */
la_status la_pcg_adjoint(la_pcg_t s, const double *g, const double *u,
                         double *dl_db, double *dl_dvalues, double rtol,
                         int maxit, la_pcg_info *info, la_stream_t stream);
/* Whether the solver fuses the step after each SpMV (no reference
 * counterpart): *fused = 1 when (p, A p), alpha, the x / r update and
 * ||r||^2 run in one cooperative kernel that finishes its own dot products,
 * 0 for separate dot and update launches (set LA_PCG_FUSED=0 in the
 * environment before la_pcg_create; the iterates are the same bit for bit). */
la_status la_pcg_fused(la_pcg_t s, int *fused);
la_status la_pcg_destroy(la_pcg_t s);

#ifdef __cplusplus
}
#endif
#endif /* LA_B200_H */
