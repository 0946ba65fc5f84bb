// dropin_main.cpp -- a caller of the C++ drop-in layer (include/la_b200.hpp),
// written the way the reference's own callers use sparse_mat_op/: the
// classes and free functions of matrix_utils::b200 with host arrays.
// tests/test_dropin.py compiles it with g++ against the header, links it to
// liblab200.so and compares what it writes with the committed fixtures.
//
//   dropin_main <in.bin> <out.bin> <coo.bin>
// in.bin: int32 n, int32 nnz, ai[n+1], aj[nnz] (int32), av[nnz], x[n],
//         y0[n] (double); a square FP64 CSR with base 0.
// out.bin: records of (int32 kind: 0 int32 / 1 double, int64 count, data),
// in the order written below.  Device results are written only when a GPU
// is present; otherwise the status the device classes throw is recorded.
// coo.bin: a file in ReadFromBinaryCOO's layout, base 1.
#include "la_b200.hpp"

#include <cstdint>
#include <cstdio>
#include <sstream>
#include <vector>

namespace m = matrix_utils::b200;

// The members SPMV<> reads from a reference CSRMatrix (rows, Base(), AI(),
// AJ(), AV(); matrix_utils.hpp:37-103).
struct Csr {
  using ROWTYPE = int;
  using COLTYPE = int;
  using VALTYPE = double;
  int rows = 0;
  std::vector<int> ai, aj;
  std::vector<double> av;
  int Base() const { return 0; }
  const int *AI() const { return ai.data(); }
  const int *AJ() const { return aj.data(); }
  const double *AV() const { return av.data(); }
};

static FILE *g_out = nullptr;

static void put(const std::vector<int> &v) {
  const int32_t k = 0;
  const int64_t c = (int64_t)v.size();
  std::fwrite(&k, 4, 1, g_out);
  std::fwrite(&c, 8, 1, g_out);
  std::fwrite(v.data(), 4, v.size(), g_out);
}
static void put(const std::vector<double> &v) {
  const int32_t k = 1;
  const int64_t c = (int64_t)v.size();
  std::fwrite(&k, 4, 1, g_out);
  std::fwrite(&c, 8, 1, g_out);
  std::fwrite(v.data(), 8, v.size(), g_out);
}

// strict lower (lower = true) or upper triangle of A
static void triangle(const Csr &A, bool lower, std::vector<int> &ai, std::vector<int> &aj,
                     std::vector<double> &av) {
  ai.assign(1, 0);
  aj.clear();
  av.clear();
  for (int i = 0; i < A.rows; i++) {
    for (int k = A.ai[i]; k < A.ai[i + 1]; k++)
      if (lower ? A.aj[k] < i : A.aj[k] > i) {
        aj.push_back(A.aj[k]);
        av.push_back(A.av[k]);
      }
    ai.push_back((int)aj.size());
  }
}

int main(int argc, char **argv) {
  if (argc != 4)
    return 2;
  FILE *in = std::fopen(argv[1], "rb");
  if (!in)
    return 2;
  int32_t n = 0, nnz = 0;
  if (std::fread(&n, 4, 1, in) != 1 || std::fread(&nnz, 4, 1, in) != 1)
    return 2;
  Csr A;
  A.rows = n;
  A.ai.resize(n + 1);
  A.aj.resize(nnz);
  A.av.resize(nnz);
  std::vector<double> x(n), y0(n);
  size_t got = std::fread(A.ai.data(), 4, n + 1, in) + std::fread(A.aj.data(), 4, nnz, in) +
               std::fread(A.av.data(), 8, nnz, in) + std::fread(x.data(), 8, n, in) +
               std::fread(y0.data(), 8, n, in);
  std::fclose(in);
  if (got != (size_t)(n + 1 + 2 * nnz + 2 * n))
    return 2;
  g_out = std::fopen(argv[2], "wb");
  if (!g_out)
    return 2;

  std::vector<int> l_ai, l_aj, u_ai, u_aj;
  std::vector<double> l_av, u_av;
  triangle(A, true, l_ai, l_aj, l_av);
  triangle(A, false, u_ai, u_aj, u_av);

  // host steps: TopologicalSort2 / TopologicalSort on L, Diagonal, permute
  std::vector<int> iperm, prefix;
  const int lv = m::TopologicalSort2<m::L>(n, 0, l_ai.data(), l_aj.data(), iperm, prefix);
  put(std::vector<int>{lv});
  put(iperm);
  put(prefix);
  std::vector<int> kip, kpf;
  const int last = m::TopologicalSort<m::L>(n, 0, l_ai.data(), l_aj.data(), kip, kpf);
  put(std::vector<int>{last});
  put(kip);
  std::vector<int> dpos(n);
  std::vector<double> diag(n);
  const bool all = m::Diagonal(n, 0, A.ai.data(), A.aj.data(), A.av.data(), dpos.data(),
                               diag.data());
  put(std::vector<int>{all ? 1 : 0});
  put(diag);
  std::vector<int> rev(n), inv;
  for (int i = 0; i < n; i++)
    rev[i] = n - 1 - i;
  m::inversePermute(inv, rev, 0);
  std::vector<int> p_ai(n + 1), p_aj(nnz);
  std::vector<double> p_av(nnz);
  m::permute(n, 0, A.ai.data(), A.aj.data(), A.av.data(), rev.data(), inv.data(), p_ai.data(),
             p_aj.data(), p_av.data());
  put(p_ai);
  put(p_aj);
  put(p_av);

  // the binary COO reader, host only (utils.h:23-44)
  auto coo_records = [&]() {
    std::vector<int> cr, cc;
    std::vector<double> cv;
    auto mn = utils::b200::ReadFromBinaryCOO(std::string(argv[3]), cr, cc, cv, 1);
    put(cr);
    put(cc);
    put(cv);
    put(std::vector<int>{mn.first, mn.second});
  };

  int sms = 0;
  if (la_device_sm_count(&sms) != LA_OK || sms == 0) {
    // no device: every device class must fail loudly, with no CPU fallback
    int status = -1;
    try {
      m::SegSumSPMV<int, int, double> s(4);
      s.preprocess(n, 0, A.ai.data(), A.aj.data(), A.av.data());
    } catch (const m::Error &e) {
      status = (int)e.status;
    }
    put(std::vector<int>{status});
    coo_records();
    std::fclose(g_out);
    return 0;
  }
  put(std::vector<int>{-1});
  coo_records();

  // SpMV: both forms and the SPMV<> adapter, y = 1.5 A x + 0.5 y0
  std::vector<double> y = y0;
  m::SegSumSPMV<int, int, double> seg(8);
  seg.preprocess(n, 0, A.ai.data(), A.aj.data(), A.av.data());
  seg(n, 0, A.ai.data(), A.aj.data(), A.av.data(), x.data(), y.data(), 1.5, 0.5);
  put(y);
  y = y0;
  m::ALBUSSPMV<int, int, double> alb(8);
  alb(n, 0, A.ai.data(), A.aj.data(), A.av.data(), x.data(), y.data(), 1.5, 0.5);
  put(y);
  y = y0;
  m::SPMV<Csr, m::SegSumSPMV<int, int, double>> ad;
  ad.setMatrix(&A);
  ad.preprocess();
  ad(x.data(), y.data(), 1.5, 0.5);
  put(y);

  // triangular solves with b = ones: strict L (unit), strict U with A's
  // diagonal, through the class and the free functions
  std::vector<double> ones(n, 1.0), t(n);
  m::OptimizedTriangularSolve<m::FBSubstitutionType::Barrier, m::L> ls(8);
  ls.analysis(n, 0, l_ai.data(), l_aj.data(), l_av.data());
  ls(ones.data(), t.data());
  put(t);
  m::OptimizedTriangularSolve<m::FBSubstitutionType::NoBarrier, m::U> us(8);
  us.analysis(n, 0, u_ai.data(), u_aj.data(), u_av.data(), diag.data());
  us(ones.data(), t.data());
  put(t);
  m::ForwardSubstitution(n, 0, l_ai.data(), l_aj.data(), l_av.data(), ones.data(), t.data());
  put(t);
  m::BackwardSubstitution(n, 0, u_ai.data(), u_aj.data(), u_av.data(), diag.data(), ones.data(),
                          t.data());
  put(t);
  m::LevelScheduleForwardSubstitution(iperm.data(), prefix.data(), lv, n, 0, l_ai.data(),
                                      l_aj.data(), l_av.data(), ones.data(), t.data());
  put(t);
  std::vector<int> uip, upf;
  const int ulv = m::TopologicalSort2<m::U>(n, 0, u_ai.data(), u_aj.data(), uip, upf);
  m::LevelScheduleBackwardSubstitution(uip.data(), upf.data(), ulv, n, 0, u_ai.data(),
                                       u_aj.data(), u_av.data(), diag.data(), ones.data(),
                                       t.data());
  put(t);
  m::ForwardSubstitutionT(n, 0, u_ai.data(), u_aj.data(), u_av.data(), ones.data(), t.data());
  put(t);

  // ReadFromBinaryCSR (utils.h:46-91) and read_matrix_market_csr
  // (utils.h:93-132), built on the device
  std::vector<int> bai, baj;
  std::vector<double> bav;
  auto bmn = utils::b200::ReadFromBinaryCSR(std::string(argv[3]), bai, baj, bav, 1);
  put(bai);
  put(baj);
  put(bav);
  put(std::vector<int>{bmn.first, bmn.second});
  std::ostringstream mm;
  mm.precision(17);
  mm << "%%MatrixMarket matrix coordinate real general\n" << n << " " << n << " " << nnz << "\n";
  for (int i = n - 1; i >= 0; i--) // rows in reverse: the reader sorts them
    for (int k = A.ai[i]; k < A.ai[i + 1]; k++)
      mm << i + 1 << " " << A.aj[k] + 1 << " " << A.av[k] << "\n";
  std::istringstream in_mm(mm.str());
  std::vector<int> mai, maj;
  std::vector<double> mav;
  utils::b200::read_matrix_market_csr(in_mm, mai, maj, mav);
  put(mai);
  put(maj);
  put(mav);
  std::fclose(g_out);
  return 0;
}
