// la_ingest.cu -- the on-disk formats either side of the path, read into a
// device CSR.
//
// Reference: utils/utils.h:23-44 ReadFromBinaryCOO (an int64 count, then one
// std::tuple<int32 row, int32 col, double value> per entry, indices carrying
// the file's base; rows / cols = largest index + 1 - base), utils.h:46-91
// ReadFromBinaryCSR (those entries sorted by (row, col), row pointers built
// with the same base) and utils.h:93-132 read_matrix_market_csr (a Matrix
// Market coordinate file through fast_matrix_market, 0-based, sorted by (row,
// col)).
//
// B200 design.  The host only parses (a binary file is a memcpy of records,
// a text file is cut at line boundaries and parsed by all host threads); the
// entries then go to the device, where a stable least-significant-digit radix
// sort orders them by (row, col) -- column digits first, then row digits,
// 8 bits per pass, only as many passes as the index ranges need, skipped
// altogether when the input is already in order -- and the row pointers are
// found by one binary search per row in the sorted rows.  Entries with equal
// (row, col) keep their input order (the reference's std::sort leaves their
// order unspecified; duplicates are kept, as the reference keeps them).
//
// Roofline: HBM-bound; each sort pass reads a 4-byte digit key per entry for
// the histogram and moves 12 bytes per entry (row, col, position).

#include "la_device.cuh"
#include "la_internal.h"

#include <algorithm>
#include <charconv>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <memory>
#include <string>
#include <vector>

#include <omp.h>

namespace la {
namespace {

constexpr int kSortThreads = 256;
constexpr int kSortChunks = 16; // 256-entry chunks per block
constexpr int kSortTile = kSortThreads * kSortChunks;
constexpr int kRadix = 256;
constexpr int kWarps = kSortThreads / 32;

// is the input already ordered by (row, col)?  flag = 1 if some neighbour
// pair is out of order
// (one store per warp that saw a pair out of order: a store per pair made
// every thread of a shuffled input write the same word)
__global__ void order_check_kernel(const long long nnz, const unsigned *row, const unsigned *col,
                                   int *flag) {
  bool out_of_order = false;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i + 1 < nnz;
       i += (long long)gridDim.x * blockDim.x) {
    const unsigned r0 = row[i], r1 = row[i + 1];
    out_of_order |= r0 > r1 || (r0 == r1 && col[i] > col[i + 1]);
  }
  if (__any_sync(0xffffffffu, out_of_order) && (threadIdx.x & 31) == 0)
    *flag = 1;
}

__device__ __forceinline__ int digit_of(unsigned key, int shift) { return (key >> shift) & 255; }

// per-block histogram of one digit; table[d * nblocks + b]
__global__ void __launch_bounds__(kSortThreads)
    radix_hist_kernel(const int nnz, const unsigned *key, const int shift, int *table) {
  __shared__ int cnt[kRadix];
  cnt[threadIdx.x] = 0;
  __syncthreads();
  const int b = blockIdx.x, base = b * kSortTile;
  for (int c = 0; c < kSortChunks; c++) {
    const int i = base + c * kSortThreads + threadIdx.x;
    if (i < nnz)
      atomicAdd(&cnt[digit_of(key[i], shift)], 1);
  }
  __syncthreads();
  table[threadIdx.x * gridDim.x + b] = cnt[threadIdx.x];
}

// Stable scatter: a block walks its tile in 256-entry chunks in index order;
// an entry's place is the digit's global offset for this block (scanned
// table) + entries of that digit earlier in the tile: earlier chunks (the
// running count), earlier warps of this chunk, earlier lanes of its warp.
__global__ void __launch_bounds__(kSortThreads)
    radix_scatter_kernel(const int nnz, const unsigned *key, const int shift,
                         const int *table, const unsigned *row_in, const unsigned *col_in,
                         const int *pos_in, unsigned *row_out, unsigned *col_out, int *pos_out) {
  __shared__ int run[kRadix];
  __shared__ int wcnt[kWarps][kRadix];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int b = blockIdx.x, base = b * kSortTile;
  run[tid] = table[tid * gridDim.x + b];
  for (int w = 0; w < kWarps; w++)
    wcnt[w][tid] = 0;
  __syncthreads();
  const unsigned lt = (1u << lane) - 1u;
  for (int c = 0; c < kSortChunks; c++) {
    const int i = base + c * kSortThreads + tid;
    const bool valid = i < nnz;
    const int d = valid ? digit_of(key[i], shift) : kRadix; // kRadix: no entry
    const unsigned same = __match_any_sync(0xffffffffu, d);
    const int rank = __popc(same & lt);
    if (valid && rank == 0)
      wcnt[warp][d] = __popc(same);
    __syncthreads();
    if (valid) {
      int pre = run[d];
      for (int w = 0; w < warp; w++)
        pre += wcnt[w][d];
      const int o = pre + rank;
      row_out[o] = row_in[i];
      col_out[o] = col_in[i];
      pos_out[o] = pos_in[i];
    }
    __syncthreads();
    int add = 0;
    for (int w = 0; w < kWarps; w++) {
      add += wcnt[w][tid];
      wcnt[w][tid] = 0;
    }
    run[tid] += add;
    __syncthreads();
  }
}

// Exclusive scan of 2048-entry chunks (2 per thread), chunk totals to sums.
constexpr int kScanThreads = 1024;
constexpr int kScanChunk = 2 * kScanThreads;

__global__ void __launch_bounds__(kScanThreads)
    scan_chunk_kernel(int *d, const int m, int *sums) {
  __shared__ int wsum[kScanThreads / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const long long i0 = (long long)blockIdx.x * kScanChunk + 2 * tid;
  const int a = i0 < m ? d[i0] : 0, b = i0 + 1 < m ? d[i0 + 1] : 0;
  int v = a + b, incl = v;
#pragma unroll
  for (int k = 1; k < 32; k <<= 1) {
    const int u = __shfl_up_sync(0xffffffffu, incl, k);
    if (lane >= k)
      incl += u;
  }
  if (lane == 31)
    wsum[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    int w = wsum[lane], wi = w;
#pragma unroll
    for (int k = 1; k < 32; k <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, wi, k);
      if (lane >= k)
        wi += u;
    }
    wsum[lane] = wi - w; // exclusive prefix of the warps' totals
    if (lane == 31 && sums)
      sums[blockIdx.x] = wi;
  }
  __syncthreads();
  const int ex = wsum[warp] + incl - v;
  if (i0 < m)
    d[i0] = ex;
  if (i0 + 1 < m)
    d[i0 + 1] = ex + a;
}

__global__ void scan_add_kernel(int *d, const int m, const int *sums) {
  const long long i = (long long)blockIdx.x * kScanChunk + threadIdx.x;
  const int add = sums[blockIdx.x];
  if (i < m)
    d[i] += add;
  if (i + kScanThreads < m && threadIdx.x + kScanThreads < kScanChunk)
    d[i + kScanThreads] += add;
}

} // namespace

la_status scan_exclusive(int *d, int m, cudaStream_t st) {
  if (m <= 0)
    return LA_OK;
  const int nb = (m + kScanChunk - 1) / kScanChunk;
  if (nb == 1) {
    scan_chunk_kernel<<<1, kScanThreads, 0, st>>>(d, m, nullptr);
    LA_CUDA_TRY(cudaGetLastError());
    return LA_OK;
  }
  DevBuf sums;
  LA_TRY(sums.alloc(sizeof(int) * nb));
  scan_chunk_kernel<<<nb, kScanThreads, 0, st>>>(d, m, sums.as<int>());
  LA_CUDA_TRY(cudaGetLastError());
  LA_TRY(scan_exclusive(sums.as<int>(), nb, st));
  scan_add_kernel<<<nb, kScanThreads, 0, st>>>(d, m, sums.as<int>());
  LA_CUDA_TRY(cudaGetLastError());
  LA_CUDA_TRY(cudaStreamSynchronize(st)); // sums is released on return
  return LA_OK;
}

namespace {

// ai[r] = base + (entries with row < r): lower bound of r in the sorted rows
__global__ void row_pointer_kernel(const int n, const int nnz, const unsigned *row,
                                   const int base, int *ai) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r > n)
    return;
  int lo = 0, hi = nnz;
  while (lo < hi) {
    const int mid = lo + ((hi - lo) >> 1);
    if (row[mid] < (unsigned)r)
      lo = mid + 1;
    else
      hi = mid;
  }
  ai[r] = base + lo;
}

template <typename V>
__global__ void gather_kernel(const int nnz, const int *pos, const unsigned *col, const int base,
                              const V *vin, int *aj, V *vout) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nnz; i += gridDim.x * blockDim.x) {
    aj[i] = int(col[i]) + base;
    vout[i] = vin[pos[i]];
  }
}

__global__ void iota_kernel(const int nnz, int *pos) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nnz; i += gridDim.x * blockDim.x)
    pos[i] = i;
}

int bits_for(unsigned range) { // bits to hold 0 .. range - 1
  int b = 0;
  while (b < 32 && (range - 1u) >> b)
    b++;
  return range <= 1 ? 0 : b;
}

} // namespace

// Stable LSD radix sort of n entries by (hi, lo), hi major: lo digits first,
// then hi digits, 8 bits per pass, as many passes as [0, hi_range) and
// [0, lo_range) need; pos travels with the keys.  Buffers [cur] hold the
// input; on return *cur names the buffers holding the result.
la_status radix_sort_pairs(int n, unsigned hi_range, unsigned lo_range, DevBuf (&kh)[2],
                           DevBuf (&kl)[2], DevBuf (&kp)[2], int *cur, cudaStream_t st) {
  if (n <= 1)
    return LA_OK;
  const int nb = (n + kSortTile - 1) / kSortTile;
  DevBuf table;
  LA_TRY(table.alloc(sizeof(int) * (size_t)kRadix * nb));
  const int lpass = (bits_for(lo_range) + 7) / 8, hpass = (bits_for(hi_range) + 7) / 8;
  int c = *cur;
  for (int pass = 0; pass < lpass + hpass; pass++) {
    const bool on_lo = pass < lpass;
    const int shift = 8 * (on_lo ? pass : pass - lpass);
    const unsigned *key = on_lo ? kl[c].as<unsigned>() : kh[c].as<unsigned>();
    radix_hist_kernel<<<nb, kSortThreads, 0, st>>>(n, key, shift, table.as<int>());
    LA_CUDA_TRY(cudaGetLastError());
    LA_TRY(scan_exclusive(table.as<int>(), kRadix * nb, st));
    radix_scatter_kernel<<<nb, kSortThreads, 0, st>>>(
        n, key, shift, table.as<int>(), kh[c].as<unsigned>(), kl[c].as<unsigned>(),
        kp[c].as<int>(), kh[1 - c].as<unsigned>(), kl[1 - c].as<unsigned>(), kp[1 - c].as<int>());
    LA_CUDA_TRY(cudaGetLastError());
    c = 1 - c;
  }
  LA_CUDA_TRY(cudaStreamSynchronize(st)); // table is released on return
  *cur = c;
  return LA_OK;
}

// out[q] = base + (number of sorted keys below q), q in [0, nq]: the start of
// every key's run in a sorted array (row pointers, level boundaries).
la_status run_starts(int n, const unsigned *sorted, int nq, int base, int *out, cudaStream_t st) {
  row_pointer_kernel<<<(nq + 1 + 255) / 256, 256, 0, st>>>(nq, n, sorted, base, out);
  LA_CUDA_TRY(cudaGetLastError());
  return LA_OK;
}

// Device CSR from host COO entries (indices carry `base`; rows[k] - base in
// [0, nrows), cols[k] - base in [0, ncols)).
la_status csr_from_coo(int nrows, int ncols, long long nnz_l, int base, const int *rows,
                       const int *cols, const void *vals, la_dtype dtype, int flags,
                       la_csr_t *out) {
  const int nnz = (int)nnz_l;
  std::vector<unsigned> r0(nnz), c0(nnz);
  bool bad = false;
#pragma omp parallel for reduction(|| : bad)
  for (int k = 0; k < nnz; k++) {
    const long long r = (long long)rows[k] - base, c = (long long)cols[k] - base;
    bad = bad || r < 0 || r >= nrows || c < 0 || c >= ncols;
    r0[k] = (unsigned)r;
    c0[k] = (unsigned)c;
  }
  if (bad) {
    set_error("COO entry index outside [base, base + rows/cols)");
    return LA_ERR_INVALID_ARG;
  }
  LA_TRY(require_device());
  std::unique_ptr<la_csr_s> A(new la_csr_s());
  A->n = nrows;
  A->ncols = ncols;
  A->nnz = nnz;
  A->base = base;
  A->dtype = dtype;
  const size_t vs = dtype == LA_F64 ? 8 : 4;
  LA_TRY(A->ai.alloc(sizeof(int) * (nrows + 1)));
  LA_TRY(A->aj.alloc(sizeof(int) * std::max(nnz, 1)));
  LA_TRY(A->av.alloc(vs * std::max(nnz, 1)));
  cudaStream_t st = nullptr;
  DevBuf kr[2], kc[2], kp[2], vin, flag;
  for (int s = 0; s < 2; s++) {
    LA_TRY(kr[s].alloc(sizeof(unsigned) * std::max(nnz, 1)));
    LA_TRY(kc[s].alloc(sizeof(unsigned) * std::max(nnz, 1)));
    LA_TRY(kp[s].alloc(sizeof(int) * std::max(nnz, 1)));
  }
  LA_TRY(vin.alloc(vs * std::max(nnz, 1)));
  LA_TRY(flag.alloc(sizeof(int)));
  if (nnz) {
    LA_CUDA_TRY(cudaMemcpyAsync(kr[0].p, r0.data(), sizeof(unsigned) * nnz,
                                cudaMemcpyHostToDevice, st));
    LA_CUDA_TRY(cudaMemcpyAsync(kc[0].p, c0.data(), sizeof(unsigned) * nnz,
                                cudaMemcpyHostToDevice, st));
    LA_CUDA_TRY(cudaMemcpyAsync(vin.p, vals, vs * nnz, cudaMemcpyHostToDevice, st));
  }
  const int g = std::max(1, std::min((nnz + 255) / 256, 16 * sm_count()));
  iota_kernel<<<g, 256, 0, st>>>(nnz, kp[0].as<int>());
  LA_CUDA_TRY(cudaMemsetAsync(flag.p, 0, sizeof(int), st));
  order_check_kernel<<<g, 256, 0, st>>>(nnz, kr[0].as<unsigned>(), kc[0].as<unsigned>(),
                                        flag.as<int>());
  LA_CUDA_TRY(cudaGetLastError());
  int unordered = 0;
  LA_CUDA_TRY(cudaMemcpy(&unordered, flag.p, sizeof(int), cudaMemcpyDeviceToHost));
  int cur = 0;
  if (unordered)
    LA_TRY(radix_sort_pairs(nnz, (unsigned)nrows, (unsigned)ncols, kr, kc, kp, &cur, st));
  row_pointer_kernel<<<(nrows + 1 + 255) / 256, 256, 0, st>>>(nrows, nnz, kr[cur].as<unsigned>(),
                                                              base, A->ai.as<int>());
  if (dtype == LA_F64)
    gather_kernel<double><<<g, 256, 0, st>>>(nnz, kp[cur].as<int>(), kc[cur].as<unsigned>(), base,
                                             vin.as<double>(), A->aj.as<int>(), A->av.as<double>());
  else
    gather_kernel<float><<<g, 256, 0, st>>>(nnz, kp[cur].as<int>(), kc[cur].as<unsigned>(), base,
                                            vin.as<float>(), A->aj.as<int>(), A->av.as<float>());
  LA_CUDA_TRY(cudaGetLastError());
  A->h_ai.resize(nrows + 1);
  LA_CUDA_TRY(cudaMemcpy(A->h_ai.data(), A->ai.p, sizeof(int) * (nrows + 1),
                         cudaMemcpyDeviceToHost));
  LA_TRY(csr_finish(A.get(), flags));
  *out = A.release();
  return LA_OK;
}

// ------------------------------------------------------------------ readers
la_status read_file(const char *path, std::string &buf) {
  std::ifstream f(path, std::ios::binary);
  if (!f) {
    set_error("cannot open '%s'", path);
    return LA_ERR_INVALID_ARG;
  }
  f.seekg(0, std::ios::end);
  const std::streamoff len = f.tellg();
  f.seekg(0, std::ios::beg);
  buf.resize((size_t)std::max<std::streamoff>(len, 0));
  if (len > 0 && !f.read(&buf[0], len)) {
    set_error("cannot read '%s'", path);
    return LA_ERR_INVALID_ARG;
  }
  return LA_OK;
}

// ReadFromBinaryCOO's records: std::tuple<int32, int32, double> as
// libstdc++ lays a tuple out (last element first): value at byte 0, column
// at byte 8, row at byte 12; 16 bytes per record.
la_status read_binary_coo(const char *path, int base, std::vector<int> &rows,
                          std::vector<int> &cols, std::vector<double> &vals, int *m, int *n) {
  std::string buf;
  LA_TRY(read_file(path, buf));
  if (buf.size() < 8) {
    set_error("'%s': shorter than the 8-byte entry count", path);
    return LA_ERR_INVALID_ARG;
  }
  long long size = 0;
  std::memcpy(&size, buf.data(), 8);
  if (size < 0 || size >= (1LL << 31) || (unsigned long long)buf.size() < 8 + 16ULL * size) {
    set_error("'%s': entry count %lld does not fit the file", path, size);
    return LA_ERR_INVALID_ARG;
  }
  rows.resize(size);
  cols.resize(size);
  vals.resize(size);
  int mr = 0, mc = 0;
  const char *p = buf.data() + 8;
#pragma omp parallel for reduction(max : mr, mc)
  for (long long k = 0; k < size; k++) {
    double v;
    int c, r;
    std::memcpy(&v, p + 16 * k, 8);
    std::memcpy(&c, p + 16 * k + 8, 4);
    std::memcpy(&r, p + 16 * k + 12, 4);
    rows[k] = r;
    cols[k] = c;
    vals[k] = v;
    mr = std::max(mr, r);
    mc = std::max(mc, c);
  }
  *m = mr + (1 - base);
  *n = mc + (1 - base);
  return LA_OK;
}

namespace {
bool ieq_prefix(const char *a, const char *b) { // does a start with b (case-insensitive)?
  for (; *b; a++, b++)
    if (std::tolower((unsigned char)*a) != std::tolower((unsigned char)*b))
      return false;
  return true;
}
const char *skip_ws(const char *p, const char *e) {
  while (p < e && (*p == ' ' || *p == '\t' || *p == '\r'))
    p++;
  return p;
}
} // namespace

// Matrix Market coordinate text (real / integer / pattern; general,
// symmetric or skew-symmetric; symmetric entries mirrored as
// fast_matrix_market's generalize_symmetry does).  0-based output.
la_status parse_matrix_market(const char *text, size_t len, std::vector<int> &rows,
                              std::vector<int> &cols, std::vector<double> &vals, int *m,
                              int *n) {
  const char *p = text, *e = text + len;
  const char *nl = (const char *)std::memchr(p, '\n', e - p);
  const std::string banner(p, nl ? nl : e);
  if (!ieq_prefix(banner.c_str(), "%%MatrixMarket")) {
    set_error("Matrix Market: missing %%%%MatrixMarket banner");
    return LA_ERR_INVALID_ARG;
  }
  std::string lower(banner);
  for (char &c : lower)
    c = (char)std::tolower((unsigned char)c);
  if (lower.find("coordinate") == std::string::npos) {
    set_error("Matrix Market: only the coordinate format is read");
    return LA_ERR_INVALID_ARG;
  }
  const bool pattern = lower.find("pattern") != std::string::npos;
  if (lower.find("complex") != std::string::npos) {
    set_error("Matrix Market: complex values are not supported");
    return LA_ERR_INVALID_ARG;
  }
  const bool skew = lower.find("skew-symmetric") != std::string::npos;
  const bool sym = skew || lower.find("symmetric") != std::string::npos ||
                   lower.find("hermitian") != std::string::npos;
  p = nl ? nl + 1 : e;
  // comments, then the size line
  long long M = -1, N = -1, NNZ = -1;
  while (p < e) {
    const char *le = (const char *)std::memchr(p, '\n', e - p);
    if (!le)
      le = e;
    const char *q = skip_ws(p, le);
    if (q < le && *q != '%') {
      auto r1 = std::from_chars(q, le, M);
      q = skip_ws(r1.ptr, le);
      auto r2 = std::from_chars(q, le, N);
      q = skip_ws(r2.ptr, le);
      auto r3 = std::from_chars(q, le, NNZ);
      if (r1.ec != std::errc() || r2.ec != std::errc() || r3.ec != std::errc()) {
        set_error("Matrix Market: bad size line");
        return LA_ERR_INVALID_ARG;
      }
      p = le < e ? le + 1 : e;
      break;
    }
    p = le < e ? le + 1 : e;
  }
  if (M < 0 || N < 0 || NNZ < 0 || M >= (1LL << 31) || N >= (1LL << 31) || NNZ >= (1LL << 30)) {
    set_error("Matrix Market: missing or out-of-range size line");
    return LA_ERR_INVALID_ARG;
  }
  // entry lines, cut into per-thread ranges at line boundaries
  const int T = std::max(1, omp_get_max_threads());
  std::vector<const char *> cut(T + 1);
  cut[0] = p;
  cut[T] = e;
  for (int t = 1; t < T; t++) {
    const char *c = p + (size_t)(e - p) * t / T;
    c = std::max(c, cut[t - 1]);
    const char *q = (const char *)std::memchr(c, '\n', e - c);
    cut[t] = q ? q + 1 : e;
  }
  std::vector<std::vector<int>> R(T), Cc(T);
  std::vector<std::vector<double>> Vv(T);
  std::vector<int> err(T, 0);
#pragma omp parallel for num_threads(T) schedule(static, 1)
  for (int t = 0; t < T; t++) {
    const char *q = cut[t], *qe = cut[t + 1];
    while (q < qe) {
      const char *le = (const char *)std::memchr(q, '\n', qe - q);
      if (!le)
        le = qe;
      const char *s = skip_ws(q, le);
      if (s < le && *s != '%') {
        long long i = 0, j = 0;
        double v = 1.0;
        auto a = std::from_chars(s, le, i);
        s = skip_ws(a.ptr, le);
        auto b = std::from_chars(s, le, j);
        s = skip_ws(b.ptr, le);
        bool ok = a.ec == std::errc() && b.ec == std::errc();
        if (ok && !pattern) {
          auto c = std::from_chars(s, le, v);
          ok = c.ec == std::errc();
        }
        if (!ok || i < 1 || i > M || j < 1 || j > N) {
          err[t] = 1;
          break;
        }
        R[t].push_back((int)(i - 1));
        Cc[t].push_back((int)(j - 1));
        Vv[t].push_back(v);
        if (sym && i != j) {
          R[t].push_back((int)(j - 1));
          Cc[t].push_back((int)(i - 1));
          Vv[t].push_back(skew ? -v : v);
        }
      }
      q = le < qe ? le + 1 : qe;
    }
  }
  for (int t = 0; t < T; t++)
    if (err[t]) {
      set_error("Matrix Market: malformed or out-of-range entry line");
      return LA_ERR_INVALID_ARG;
    }
  size_t total = 0;
  for (int t = 0; t < T; t++)
    total += R[t].size();
  rows.clear();
  cols.clear();
  vals.clear();
  rows.reserve(total);
  cols.reserve(total);
  vals.reserve(total);
  for (int t = 0; t < T; t++) {
    rows.insert(rows.end(), R[t].begin(), R[t].end());
    cols.insert(cols.end(), Cc[t].begin(), Cc[t].end());
    vals.insert(vals.end(), Vv[t].begin(), Vv[t].end());
  }
  *m = (int)M;
  *n = (int)N;
  return LA_OK;
}

} // namespace la
