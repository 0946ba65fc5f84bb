// la_rcm.cu -- the Cuthill-McKee ordering of large components on the GPU.
//
// Reference: SerialCM (reordering/Reordering.cpp:37-136) with its
// PseudoDiameter search (reordering/Reordering.h:72-136), as la_host.cpp's
// rcm restates its observable rules: the source is the first node of
// minimum degree; a BFS from it; up to five last-level candidates taken by
// (degree, index), each candidate's and its neighbours' degrees set to
// INT_MAX (a change the sweep's ties then see); a BFS from the first
// candidate -- if deeper it becomes the source and the search repeats.  The
// Cuthill-McKee sweep then visits the ordering level by level and appends,
// for each node, its not yet claimed neighbours of the next level sorted by
// (degree, index).
//
// B200 design.  A level-synchronous BFS (a vertex is claimed by a
// compare-and-swap on its level, so the levels are the sequential search's)
// and packed (degree, index) minimum reductions give the source.  The sweep
// needs no sequential walk: a node of level l+1 is appended by the first
// node of level l, in the ordering, that neighbours it, so per level (1)
// every next-level node finds the smallest ordering position among its
// level-l neighbours (its parent), (2) every level-l node counts the
// next-level nodes it is the parent of, (3) a scan of the counts gives each
// parent's first slot, and (4) every parent sorts its children by (degree,
// index) into its slots.  The search and the sweep each run as ONE
// cooperative launch whose levels are separated by grid barriers (bounded:
// a wait that exceeds 1 s sets an error word and the launch ends), so the
// host waits once per search, not once per level.  Integer work only: the
// ordering equals the host's exactly.  Used for components of at least
// kRcmDeviceMin nodes whose rows hold at most kRcmMaxDegree entries (a
// parent's children are sorted in registers); the host orders the rest.
//
// Roofline: latency-bound (a grid barrier per BFS level, three per sweep
// level); each level reads its nodes' rows once per step.

#include "la_device.cuh"
#include "la_internal.h"

#include <algorithm>
#include <climits>
#include <cstdlib>
#include <vector>

namespace la {
namespace {

constexpr int kThreads = 256;

constexpr int kNbrGroup = 8; // neighbours whose loads are issued together

// The whole search in one cooperative launch.  Level l is queue[lstart[l],
// lstart[l+1]); at step lev the grid expands level lev-1, appending the
// vertices it claims after the frontier, then meets at a grid barrier and
// reads the new level's size.  A warp walks 32 frontier vertices together,
// kNbrGroup neighbours per vertex at a time (their column and level loads
// issued together), and appends what its lanes claimed with one atomic.
// cnt3 holds three rotating counters: the one step lev+1 uses is cleared
// during step lev, when every thread has passed the barrier after its last
// read (at step lev-2).  bar[0..2]: the barrier; bar[3]: the number of
// levels, written at the end.
__global__ void __launch_bounds__(kThreads)
    bfs_kernel(int *queue, int *level, const int *__restrict__ ai, const int *__restrict__ aj,
               const int base, int *lstart, int *cnt3, unsigned *bar) {
  const int gt = blockIdx.x * blockDim.x + threadIdx.x, gs = gridDim.x * blockDim.x;
  const int lane = threadIdx.x & 31;
  int qs = 0, qe = 1;
  for (int lev = 1;; lev++) {
    int *cnt = cnt3 + lev % 3;
    if (gt == 0)
      cnt3[(lev + 1) % 3] = 0;
    // warp-uniform walk: lane h = h0 + lane
    for (int h0 = qs + gt - lane; h0 < qe; h0 += gs) {
      const int h = h0 + lane;
      int a = 0, e = 0;
      if (h < qe) {
        const int u = __ldcg(queue + h);
        a = __ldg(ai + u) - base;
        e = __ldg(ai + u + 1) - base;
      }
      const int groups = __reduce_max_sync(0xffffffffu, (e - a + kNbrGroup - 1) / kNbrGroup);
      for (int g = 0; g < groups; g++) {
        int v[kNbrGroup], lv[kNbrGroup];
#pragma unroll
        for (int q = 0; q < kNbrGroup; q++) {
          const int k = a + g * kNbrGroup + q;
          v[q] = k < e ? __ldg(aj + k) - base : -1;
        }
#pragma unroll
        for (int q = 0; q < kNbrGroup; q++)
          lv[q] = v[q] >= 0 ? __ldcg(level + v[q]) : 0;
        int mine = 0; // claimed this round
#pragma unroll
        for (int q = 0; q < kNbrGroup; q++) {
          const bool got = v[q] >= 0 && lv[q] < 0 && atomicCAS(level + v[q], -1, lev) == -1;
          if (!got)
            v[q] = -1;
          mine += got;
        }
        int incl = mine; // warp prefix of the claims, one atomic per warp
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int t = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o)
            incl += t;
        }
        int at = 0;
        if (lane == 31 && incl > 0)
          at = atomicAdd(cnt, incl);
        at = __shfl_sync(0xffffffffu, at, 31) + incl - mine;
#pragma unroll
        for (int q = 0; q < kNbrGroup; q++)
          if (v[q] >= 0)
            queue[qe + at++] = v[q];
      }
    }
    dev::grid_barrier(bar);
    if (dev::ld_relaxed((const int *)bar + 2) != 0)
      return; // a barrier wait gave up
    const int c = dev::ld_relaxed(cnt);
    if (c == 0) {
      if (gt == 0)
        bar[3] = lev;
      return;
    }
    qs = qe;
    qe += c;
    if (gt == 0)
      lstart[lev + 1] = qe;
  }
}

// level[v] = -1 for the nodes a previous search reached
__global__ void bfs_reset_kernel(const int m, const int *queue, int *level) {
  for (int h = blockIdx.x * blockDim.x + threadIdx.x; h < m; h += gridDim.x * blockDim.x)
    level[queue[h]] = -1;
}

__global__ void bfs_start_kernel(const int src, int *queue, int *level, int *lstart) {
  queue[0] = src;
  level[src] = 0;
  lstart[0] = 0;
  lstart[1] = 1;
}

// smallest (degree, node) over list[0, m) whose degree is not INT_MAX
__global__ void argmin_kernel(const int m, const int *list, const int *deg,
                              unsigned long long *best) {
  unsigned long long b = ~0ull;
  for (int h = blockIdx.x * blockDim.x + threadIdx.x; h < m; h += gridDim.x * blockDim.x) {
    const int v = list[h];
    if (deg[v] != INT_MAX)
      b = min(b, ((unsigned long long)(unsigned)deg[v] << 32) | (unsigned)v);
  }
  for (int o = 16; o > 0; o >>= 1)
    b = min(b, __shfl_down_sync(0xffffffffu, b, o));
  if ((threadIdx.x & 31) == 0 && b != ~0ull)
    atomicMin(best, b);
}

// the search's mark: the candidate's and its neighbours' degrees -> INT_MAX
__global__ void mark_kernel(const int sel, int *deg, const int *__restrict__ ai,
                            const int *__restrict__ aj, const int base) {
  const int a = __ldg(ai + sel) - base, e = __ldg(ai + sel + 1) - base;
  if (blockIdx.x == 0 && threadIdx.x == 0)
    deg[sel] = INT_MAX;
  for (int k = a + blockIdx.x * blockDim.x + threadIdx.x; k < e; k += gridDim.x * blockDim.x)
    deg[__ldg(aj + k) - base] = INT_MAX;
}

// Exclusive scan (and total) of one value per thread over the block.
__device__ int block_exclusive_scan(int v, int *total) {
  __shared__ int wsum[kThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int incl = v;
  for (int k = 1; k < 32; k <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, incl, k);
    if (lane >= k)
      incl += t;
  }
  if (lane == 31)
    wsum[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    const int w = lane < kThreads / 32 ? wsum[lane] : 0;
    int wi = w;
    for (int k = 1; k < 32; k <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, wi, k);
      if (lane >= k)
        wi += t;
    }
    if (lane < kThreads / 32)
      wsum[lane] = wi - w;
    if (lane == kThreads / 32 - 1)
      *total = wi;
  }
  __syncthreads();
  const int ex = wsum[warp] + incl - v;
  __syncthreads(); // wsum is reused by the next call
  return ex;
}

// The Cuthill-McKee sweep in one cooperative launch, for the search whose
// level starts are lstart[0, height]; cm[0] = source and pos[source] = 0 on
// entry.  Per level l, three steps separated by grid barriers:
//  (1) parent[v] of each level-(l+1) node: the smallest ordering position
//      among its level-l neighbours;
//  (2) each level-l position p counts its children (level-(l+1) neighbours
//      whose parent is p); the counts are scanned within tiles of kThreads
//      positions (cnt) and each tile's total kept (tile_sum);
//  (4) each position's first slot is q0 + (tiles before its own) + cnt; it
//      sorts its children by (degree, node) and writes them to cm and pos.
// Arrays written inside the launch are read with __ldcg (L2, coherent).
template <int MAXC>
__global__ void __launch_bounds__(kThreads)
    cm_sweep_kernel(const int height, const int *__restrict__ lstart,
                    const int *__restrict__ queue, const int *__restrict__ level, int *pos,
                    int *parent, int *cm, int *cnt, int *tile_sum, const int *__restrict__ deg,
                    const int *__restrict__ ai, const int *__restrict__ aj, const int base,
                    unsigned *bar) {
  __shared__ int tile_total, tile_base;
  const int gt = blockIdx.x * blockDim.x + threadIdx.x, gs = gridDim.x * blockDim.x;
  for (int l = 0; l + 1 < height; l++) {
    const int p0 = __ldg(lstart + l), q0 = __ldg(lstart + l + 1);
    const int m = q0 - p0, mq = __ldg(lstart + l + 2) - q0;
    // (1) neighbours kNbrGroup at a time: columns, then levels, then the
    // positions of those on level l, each set of loads issued together
    for (int h = gt; h < mq; h += gs) {
      const int v = __ldg(queue + q0 + h);
      const int a = __ldg(ai + v) - base, e = __ldg(ai + v + 1) - base;
      int p = INT_MAX;
      for (int k0 = a; k0 < e; k0 += kNbrGroup) {
        int u[kNbrGroup], pu[kNbrGroup];
#pragma unroll
        for (int q = 0; q < kNbrGroup; q++)
          u[q] = k0 + q < e ? __ldg(aj + k0 + q) - base : -1;
#pragma unroll
        for (int q = 0; q < kNbrGroup; q++)
          if (u[q] >= 0 && __ldg(level + u[q]) != l)
            u[q] = -1;
#pragma unroll
        for (int q = 0; q < kNbrGroup; q++)
          pu[q] = u[q] >= 0 ? __ldcg(pos + u[q]) : INT_MAX;
#pragma unroll
        for (int q = 0; q < kNbrGroup; q++)
          p = min(p, pu[q]);
      }
      parent[v] = p;
    }
    dev::grid_barrier(bar);
    if (dev::ld_relaxed((const int *)bar + 2) != 0)
      return;
    // (2)
    const int ntiles = (m + kThreads - 1) / kThreads;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
      const int h = t * kThreads + threadIdx.x;
      int c = 0;
      if (h < m) {
        const int p = p0 + h, u = __ldcg(cm + p);
        const int a = __ldg(ai + u) - base, e = __ldg(ai + u + 1) - base;
        for (int k0 = a; k0 < e; k0 += kNbrGroup) {
          int v[kNbrGroup];
#pragma unroll
          for (int q = 0; q < kNbrGroup; q++)
            v[q] = k0 + q < e ? __ldg(aj + k0 + q) - base : -1;
#pragma unroll
          for (int q = 0; q < kNbrGroup; q++)
            if (v[q] >= 0 && __ldg(level + v[q]) != l + 1)
              v[q] = -1;
#pragma unroll
          for (int q = 0; q < kNbrGroup; q++)
            c += v[q] >= 0 && __ldcg(parent + v[q]) == p;
        }
      }
      const int ex = block_exclusive_scan(c, &tile_total);
      if (h < m)
        cnt[h] = ex;
      if (threadIdx.x == 0)
        tile_sum[t] = tile_total;
    }
    dev::grid_barrier(bar);
    if (dev::ld_relaxed((const int *)bar + 2) != 0)
      return;
    // (4)
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
      int s = 0;
      for (int k = threadIdx.x; k < t; k += kThreads)
        s += __ldcg(tile_sum + k);
      block_exclusive_scan(s, &tile_base);
      const int h = t * kThreads + threadIdx.x;
      if (h < m) {
        const int p = p0 + h, u = __ldcg(cm + p);
        const int a = __ldg(ai + u) - base, e = __ldg(ai + u + 1) - base;
        int ch[MAXC], cd[MAXC]; // children and their degrees, by (degree, node)
        int c = 0;
        for (int k0 = a; k0 < e; k0 += kNbrGroup) {
          int v[kNbrGroup], dv[kNbrGroup];
#pragma unroll
          for (int q = 0; q < kNbrGroup; q++)
            v[q] = k0 + q < e ? __ldg(aj + k0 + q) - base : -1;
#pragma unroll
          for (int q = 0; q < kNbrGroup; q++)
            if (v[q] >= 0 && __ldg(level + v[q]) != l + 1)
              v[q] = -1;
#pragma unroll
          for (int q = 0; q < kNbrGroup; q++)
            if (v[q] >= 0 && __ldcg(parent + v[q]) != p)
              v[q] = -1;
#pragma unroll
          for (int q = 0; q < kNbrGroup; q++)
            dv[q] = v[q] >= 0 ? __ldg(deg + v[q]) : 0;
#pragma unroll
          for (int q = 0; q < kNbrGroup; q++) {
            if (v[q] < 0 || c >= MAXC)
              continue;
            int i = c++; // insertion by (degree, node)
            while (i > 0 && (cd[i - 1] > dv[q] || (cd[i - 1] == dv[q] && ch[i - 1] > v[q]))) {
              ch[i] = ch[i - 1];
              cd[i] = cd[i - 1];
              i--;
            }
            ch[i] = v[q];
            cd[i] = dv[q];
          }
        }
        const int o = q0 + tile_base + __ldcg(cnt + h);
        for (int i = 0; i < c; i++) {
          cm[o + i] = ch[i];
          pos[ch[i]] = o + i;
        }
      }
    }
    dev::grid_barrier(bar);
    if (dev::ld_relaxed((const int *)bar + 2) != 0)
      return;
  }
}

__global__ void add_base_copy_kernel(const int m, const int *cm, const int base, int *out) {
  for (int h = blockIdx.x * blockDim.x + threadIdx.x; h < m; h += gridDim.x * blockDim.x)
    out[h] = cm[h] + base;
}

int blocks_for(int m) { return std::max(1, std::min((m + kThreads - 1) / kThreads, 4096)); }

} // namespace
} // namespace la

namespace la {

struct RcmDevice {
  int n = 0, base = 0, grid = 0;
  DevBuf ai, aj, deg, level, queue, pos, parent, cm, cnt, best, count, lstart, tiles, cnt3, bar;
  cudaStream_t st = nullptr;

  la_status init(int n_, int base_, const int *h_ai, const int *h_aj, const int *h_deg) {
    n = n_;
    base = base_;
    const int nnz = h_ai[n] - base;
    LA_TRY(ai.upload(h_ai, sizeof(int) * (n + 1)));
    LA_TRY(aj.upload(h_aj, sizeof(int) * std::max(nnz, 1)));
    LA_TRY(deg.upload(h_deg, sizeof(int) * n));
    return init_work();
  }
  // a 0-based graph already on the device: its buffers are taken over
  la_status init_device(int n_, DevBuf &d_ai, DevBuf &d_aj) {
    n = n_;
    base = 0;
    std::swap(ai.p, d_ai.p);
    std::swap(ai.bytes, d_ai.bytes);
    std::swap(aj.p, d_aj.p);
    std::swap(aj.bytes, d_aj.bytes);
    return init_work();
  }
  la_status init_work() {
    for (DevBuf *b : {&level, &queue, &pos, &parent, &cm, &cnt})
      LA_TRY(b->alloc(sizeof(int) * n));
    LA_TRY(lstart.alloc(sizeof(int) * (n + 2)));
    LA_TRY(tiles.alloc(sizeof(int) * (n / kThreads + 2)));
    LA_TRY(cnt3.alloc(sizeof(int) * 3));
    LA_TRY(bar.alloc(sizeof(unsigned) * 4));
    LA_TRY(best.alloc(sizeof(unsigned long long)));
    LA_TRY(count.alloc(sizeof(int)));
    LA_CUDA_TRY(cudaMemset(level.p, 0xff, sizeof(int) * n));
    // Cooperative grid: LA_RCM_CTAS_PER_SM CTAs per SM (tuning override;
    // default 2), capped by what fits for both kernels.  A level is a few
    // thousand to a few hundred thousand nodes; more CTAs only lengthen the
    // barriers.
    int fit = 1 << 30;
    for (const void *f : {(const void *)bfs_kernel,
                          (const void *)cm_sweep_kernel<kRcmMaxDegree>}) {
      int per_sm = 0;
      LA_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, f, kThreads, 0));
      fit = std::min(fit, per_sm);
    }
    if (fit < 1) {
      set_error("RCM: the cooperative kernels do not fit on an SM");
      return LA_ERR_CUDA;
    }
    int want = 2;
    if (const char *e = std::getenv("LA_RCM_CTAS_PER_SM"))
      want = std::max(1, std::atoi(e));
    grid = std::min(want, fit) * sm_count();
    return LA_OK;
  }

  la_status barrier_status() {
    unsigned b[4];
    LA_CUDA_TRY(cudaMemcpyAsync(b, bar.p, sizeof(b), cudaMemcpyDeviceToHost, st));
    LA_CUDA_TRY(cudaStreamSynchronize(st));
    if (b[2]) {
      set_error("RCM: a grid barrier wait exceeded its 1 s bound");
      return LA_ERR_TIMEOUT;
    }
    return LA_OK;
  }

  // BFS from src; lstart[l] = first queue slot of level l (l <= height);
  // the previous search's reached set (reached) is reset first.
  la_status bfs(int src, int &reached, std::vector<int> &ls, int *height) {
    if (reached > 0) {
      bfs_reset_kernel<<<blocks_for(reached), kThreads, 0, st>>>(reached, queue.as<int>(),
                                                                 level.as<int>());
      LA_CUDA_TRY(cudaGetLastError());
    }
    bfs_start_kernel<<<1, 1, 0, st>>>(src, queue.as<int>(), level.as<int>(), lstart.as<int>());
    LA_CUDA_TRY(cudaGetLastError());
    LA_CUDA_TRY(cudaMemsetAsync(bar.p, 0, sizeof(unsigned) * 4, st));
    LA_CUDA_TRY(cudaMemsetAsync(cnt3.p, 0, sizeof(int) * 3, st));
    int *q = queue.as<int>(), *lv = level.as<int>(), *ls_d = lstart.as<int>();
    int *c3 = cnt3.as<int>(), b = base;
    const int *dai = ai.as<int>(), *daj = aj.as<int>();
    unsigned *br = bar.as<unsigned>();
    void *args[] = {&q, &lv, &dai, &daj, &b, &ls_d, &c3, &br};
    LA_CUDA_TRY(cudaLaunchCooperativeKernel((const void *)bfs_kernel, dim3(grid),
                                            dim3(kThreads), args, 0, st));
    unsigned s4[4];
    LA_CUDA_TRY(cudaMemcpyAsync(s4, bar.p, sizeof(s4), cudaMemcpyDeviceToHost, st));
    LA_CUDA_TRY(cudaStreamSynchronize(st));
    if (s4[2]) {
      set_error("RCM: a grid barrier wait exceeded its 1 s bound");
      return LA_ERR_TIMEOUT;
    }
    const int h = (int)s4[3];
    ls.resize(h + 1);
    LA_CUDA_TRY(cudaMemcpy(ls.data(), lstart.p, sizeof(int) * (h + 1), cudaMemcpyDeviceToHost));
    reached = ls[h];
    *height = h;
    return LA_OK;
  }

  // the sweep for the last search (from src, height levels): cm, pos
  la_status sweep(int src, int height) {
    LA_CUDA_TRY(cudaMemcpyAsync(cm.p, &src, sizeof(int), cudaMemcpyHostToDevice, st));
    const int zero = 0;
    LA_CUDA_TRY(cudaMemcpyAsync(pos.as<int>() + src, &zero, sizeof(int),
                                cudaMemcpyHostToDevice, st));
    LA_CUDA_TRY(cudaMemsetAsync(bar.p, 0, sizeof(unsigned) * 4, st));
    int h = height, b = base;
    const int *ls_d = lstart.as<int>(), *q = queue.as<int>(), *lv = level.as<int>();
    int *ps = pos.as<int>(), *pa = parent.as<int>(), *c = cm.as<int>(), *ct = cnt.as<int>();
    int *ts = tiles.as<int>();
    const int *dg = deg.as<int>(), *dai = ai.as<int>(), *daj = aj.as<int>();
    unsigned *br = bar.as<unsigned>();
    void *args[] = {&h, &ls_d, &q, &lv, &ps, &pa, &c, &ct, &ts, &dg, &dai, &daj, &b, &br};
    LA_CUDA_TRY(cudaLaunchCooperativeKernel((const void *)cm_sweep_kernel<kRcmMaxDegree>,
                                            dim3(grid), dim3(kThreads), args, 0, st));
    return barrier_status();
  }

  // smallest (degree, node) among list[0, m) with degree != INT_MAX; -1 if none
  la_status argmin(const int *list, int m, int *node) {
    const unsigned long long none = ~0ull;
    LA_CUDA_TRY(cudaMemcpyAsync(best.p, &none, sizeof(none), cudaMemcpyHostToDevice, st));
    argmin_kernel<<<blocks_for(m), kThreads, 0, st>>>(m, list, deg.as<int>(),
                                                      best.as<unsigned long long>());
    LA_CUDA_TRY(cudaGetLastError());
    unsigned long long b = 0;
    LA_CUDA_TRY(cudaMemcpy(&b, best.p, sizeof(b), cudaMemcpyDeviceToHost));
    *node = b == none ? -1 : (int)(b & 0xffffffffu);
    return LA_OK;
  }
};

RcmDevice *rcm_device_create(int n, int base, const int *ai, const int *aj, const int *deg,
                             la_status *st) {
  auto *D = new RcmDevice();
  *st = D->init(n, base, ai, aj, deg);
  if (*st != LA_OK) {
    delete D;
    return nullptr;
  }
  return D;
}

void rcm_device_destroy(RcmDevice *D) { delete D; }



} // namespace la

// ---- The partitioner's landmark stage on the device: the triangle's graph
// made undirected, the breadth-first distances from up to eight landmarks
// (the first vertex of minimum degree, then farthest-point sampling over the
// vertices of minimum degree), and for every landmark pair the coordinate
// d_a - d_b: monotone along every stored entry or not, and its range.  The
// same landmarks, candidates and coordinates as la_partition.cpp's host
// stage (integer work throughout).
namespace la {
namespace {

__global__ void und_count_kernel(const int n, const int *__restrict__ ai,
                                 const int *__restrict__ aj, int *cnt) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    const int a = ai[v], e = ai[v + 1];
    atomicAdd(cnt + v, e - a);
    for (int k = a; k < e; k++)
      atomicAdd(cnt + aj[k], 1);
  }
}

__global__ void und_fill_kernel(const int n, const int *__restrict__ ai,
                                const int *__restrict__ aj, int *cursor, int *adj) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
    for (int k = ai[v]; k < ai[v + 1]; k++) {
      const int j = aj[k];
      adj[atomicAdd(cursor + v, 1)] = j;
      adj[atomicAdd(cursor + j, 1)] = v;
    }
}

__global__ void rebase_copy_kernel(const long long m, const int *in, const int base, int *out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = in[i] - base;
}

// smallest (degree, vertex)
__global__ void min_degree_kernel(const int n, const int *__restrict__ xadj,
                                  unsigned long long *best) {
  unsigned long long b = ~0ull;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
    b = min(b, ((unsigned long long)(unsigned)(xadj[v + 1] - xadj[v]) << 32) | (unsigned)v);
  for (int o = 16; o > 0; o >>= 1)
    b = min(b, __shfl_down_sync(0xffffffffu, b, o));
  if ((threadIdx.x & 31) == 0)
    atomicMin(best, b);
}

// among the vertices of degree dmin: largest mind, the smallest vertex on ties
__global__ void farthest_kernel(const int n, const int dmin, const int *__restrict__ xadj,
                                const int *__restrict__ mind, unsigned long long *best) {
  unsigned long long b = 0;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
    if (xadj[v + 1] - xadj[v] == dmin)
      b = max(b, ((unsigned long long)(unsigned)mind[v] << 32) | (0xffffffffu - (unsigned)v));
  for (int o = 16; o > 0; o >>= 1)
    b = max(b, __shfl_down_sync(0xffffffffu, b, o));
  if ((threadIdx.x & 31) == 0)
    atomicMax(best, b);
}

__global__ void min_update_kernel(const int n, const int *__restrict__ d, int *mind) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
    mind[v] = min(mind[v], d[v]);
}

constexpr int kMaxLandmarks = 8; // 28 pairs: one bit each in a 32-bit mask

// Pair p = (a, b), a < b < L, numbered (0,1), (0,2), ... as the host reads
// them.  The loops run over the compile-time maximum and test against L, so
// the per-landmark distances and per-pair extrema stay in registers.
__device__ __forceinline__ int pair_index(int L, int a, int b) {
  return a * L - a * (a + 1) / 2 + (b - a - 1);
}

// bit p of pos / neg: d_a - d_b rises / falls along some stored entry (i, j)
// of the triangle
__global__ void pair_sign_kernel(const int n, const int L, const int *__restrict__ ai,
                                 const int *__restrict__ aj, const int *__restrict__ dist,
                                 unsigned *masks) {
  unsigned pos = 0, neg = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int di[kMaxLandmarks];
#pragma unroll
    for (int l = 0; l < kMaxLandmarks; l++)
      di[l] = l < L ? __ldg(dist + (size_t)l * n + i) : 0;
    for (int k = __ldg(ai + i); k < __ldg(ai + i + 1); k++) {
      const int j = __ldg(aj + k);
      int dj[kMaxLandmarks];
#pragma unroll
      for (int l = 0; l < kMaxLandmarks; l++)
        dj[l] = l < L ? __ldg(dist + (size_t)l * n + j) : 0;
#pragma unroll
      for (int a = 0; a < kMaxLandmarks; a++)
#pragma unroll
        for (int b = a + 1; b < kMaxLandmarks; b++)
          if (b < L) {
            const int df = (di[a] - di[b]) - (dj[a] - dj[b]);
            const int p = pair_index(L, a, b);
            pos |= (unsigned)(df > 0) << p;
            neg |= (unsigned)(df < 0) << p;
          }
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    pos |= __shfl_down_sync(0xffffffffu, pos, o);
    neg |= __shfl_down_sync(0xffffffffu, neg, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicOr(masks, pos);
    atomicOr(masks + 1, neg);
  }
}

// lo[p] / hi[p]: the smallest / largest d_a - d_b over all vertices
__global__ void pair_range_kernel(const int n, const int L, const int *__restrict__ dist,
                                  int *lo, int *hi) {
  constexpr int kPairs = kMaxLandmarks * (kMaxLandmarks - 1) / 2;
  int mn[kPairs], mx[kPairs];
#pragma unroll
  for (int q = 0; q < kPairs; q++) {
    mn[q] = INT_MAX;
    mx[q] = INT_MIN;
  }
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    int d[kMaxLandmarks];
#pragma unroll
    for (int l = 0; l < kMaxLandmarks; l++)
      d[l] = l < L ? __ldg(dist + (size_t)l * n + v) : 0;
    int q = 0; // register slot: pairs of the compile-time maximum
#pragma unroll
    for (int a = 0; a < kMaxLandmarks; a++)
#pragma unroll
      for (int b = a + 1; b < kMaxLandmarks; b++, q++) {
        mn[q] = min(mn[q], d[a] - d[b]);
        mx[q] = max(mx[q], d[a] - d[b]);
      }
  }
  // warps, then the block's warps in shared memory, then one atomic per
  // pair and block (atomics from every warp on the same 56 words serialise)
  __shared__ int smn[32][kPairs], smx[32][kPairs];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < kPairs; q++) {
    int x = mn[q], y = mx[q];
    for (int o = 16; o > 0; o >>= 1) {
      x = min(x, __shfl_down_sync(0xffffffffu, x, o));
      y = max(y, __shfl_down_sync(0xffffffffu, y, o));
    }
    if (lane == 0) {
      smn[warp][q] = x;
      smx[warp][q] = y;
    }
  }
  __syncthreads();
  if (threadIdx.x < kPairs) {
    const int q = threadIdx.x;
    int x = INT_MAX, y = INT_MIN;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
      x = min(x, smn[w][q]);
      y = max(y, smx[w][q]);
    }
    int a = 0; // pair q of the compile-time maximum: pairs of a start at
               // a (2K - a - 1) / 2
    while (a + 1 < kMaxLandmarks && (a + 1) * (2 * kMaxLandmarks - a - 2) / 2 <= q)
      a++;
    const int b = a + 1 + q - a * (2 * kMaxLandmarks - a - 1) / 2;
    if (b < L) {
      atomicMin(lo + pair_index(L, a, b), x);
      atomicMax(hi + pair_index(L, a, b), y);
    }
  }
}

__global__ void coordinate_kernel(const int n, const int *__restrict__ da,
                                  const int *__restrict__ db, const int sign, int *f) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
    f[v] = sign * (da[v] - db[v]);
}

int vgrid(long long m) { return (int)std::max(1LL, std::min((m + 255) / 256, 8LL * sm_count())); }

} // namespace

struct LandmarksDevice {
  int n = 0, L = 0;
  RcmDevice D;
  DevBuf tai, taj; // the triangle, 0-based
  DevBuf dist, mind, f, scratch;
};

LandmarksDevice *landmarks_device_create(int n, int base, const int *ai, const int *aj,
                                         la_status *st) {
  auto fail = [&](LandmarksDevice *M, la_status s) {
    *st = s;
    delete M;
    return (LandmarksDevice *)nullptr;
  };
  auto *M = new LandmarksDevice();
  M->n = n;
  const long long nnz = (long long)ai[n] - base;
  DevBuf raw, xadj, adj, cursor;
  la_status s;
  if ((s = raw.upload(ai, sizeof(int) * (n + 1))) != LA_OK ||
      (s = M->tai.alloc(sizeof(int) * (n + 1))) != LA_OK)
    return fail(M, s);
  rebase_copy_kernel<<<vgrid(n + 1), 256>>>(n + 1, raw.as<int>(), base, M->tai.as<int>());
  if ((s = raw.upload(aj, sizeof(int) * std::max(nnz, 1LL))) != LA_OK ||
      (s = M->taj.alloc(sizeof(int) * std::max(nnz, 1LL))) != LA_OK)
    return fail(M, s);
  rebase_copy_kernel<<<vgrid(nnz), 256>>>(nnz, raw.as<int>(), base, M->taj.as<int>());
  raw.release();
  // the undirected graph: a row's own entries and its transpose's, any order
  if ((s = xadj.alloc(sizeof(int) * (n + 1))) != LA_OK ||
      (s = adj.alloc(sizeof(int) * std::max(2 * nnz, 1LL))) != LA_OK ||
      (s = cursor.alloc(sizeof(int) * (n + 1))) != LA_OK)
    return fail(M, s);
  if (cudaMemset(xadj.p, 0, sizeof(int) * (n + 1)) != cudaSuccess)
    return fail(M, LA_ERR_CUDA);
  und_count_kernel<<<vgrid(n), 256>>>(n, M->tai.as<int>(), M->taj.as<int>(), xadj.as<int>());
  if ((s = scan_exclusive(xadj.as<int>(), n + 1, nullptr)) != LA_OK)
    return fail(M, s);
  if (cudaMemcpy(cursor.p, xadj.p, sizeof(int) * (n + 1), cudaMemcpyDeviceToDevice) !=
      cudaSuccess)
    return fail(M, LA_ERR_CUDA);
  und_fill_kernel<<<vgrid(n), 256>>>(n, M->tai.as<int>(), M->taj.as<int>(), cursor.as<int>(),
                                     adj.as<int>());
  if (cudaGetLastError() != cudaSuccess) {
    set_error("partition landmarks: a kernel launch failed");
    return fail(M, LA_ERR_CUDA);
  }
  if ((s = M->D.init_device(n, xadj, adj)) != LA_OK)
    return fail(M, s);
  *st = LA_OK;
  return M;
}

void landmarks_device_destroy(LandmarksDevice *M) { delete M; }

la_status landmarks_device_candidates(LandmarksDevice *M, std::vector<PartitionCand> &cands) {
  const int n = M->n;
  cands.clear();
  M->L = 0;
  LA_TRY(M->dist.alloc(sizeof(int) * (size_t)n * kMaxLandmarks));
  LA_TRY(M->mind.alloc(sizeof(int) * n));
  LA_TRY(M->scratch.alloc(sizeof(unsigned long long) * 2));
  const int *xadj = M->D.ai.as<int>();
  unsigned long long *best = M->scratch.as<unsigned long long>();
  auto reduce = [&](bool farthest, int dmin, unsigned long long *out) -> la_status {
    const unsigned long long init = farthest ? 0ull : ~0ull;
    LA_CUDA_TRY(cudaMemcpy(best, &init, sizeof(init), cudaMemcpyHostToDevice));
    if (farthest)
      farthest_kernel<<<vgrid(n), 256>>>(n, dmin, xadj, M->mind.as<int>(), best);
    else
      min_degree_kernel<<<vgrid(n), 256>>>(n, xadj, best);
    LA_CUDA_TRY(cudaGetLastError());
    LA_CUDA_TRY(cudaMemcpy(out, best, sizeof(*out), cudaMemcpyDeviceToHost));
    return LA_OK;
  };
  unsigned long long key = 0;
  LA_TRY(reduce(false, 0, &key));
  const int dmin = (int)(key >> 32), v0 = (int)(key & 0xffffffffu);
  int reached = 0, height = 0;
  std::vector<int> ls;
  auto search = [&](int src, int l) -> la_status {
    LA_TRY(M->D.bfs(src, reached, ls, &height));
    // level[] holds this search's distances (-1 where unreached)
    LA_CUDA_TRY(cudaMemcpy(M->dist.as<int>() + (size_t)l * n, M->D.level.p, sizeof(int) * n,
                           cudaMemcpyDeviceToDevice));
    return LA_OK;
  };
  LA_TRY(search(v0, 0));
  if (reached != n)
    return LA_OK; // not connected: no landmark coordinates (as on the host)
  M->L = 1;
  LA_CUDA_TRY(cudaMemcpy(M->mind.p, M->dist.p, sizeof(int) * n, cudaMemcpyDeviceToDevice));
  while (M->L < kMaxLandmarks) {
    LA_TRY(reduce(true, dmin, &key));
    if ((key >> 32) == 0)
      break; // the farthest vertex of minimum degree is a landmark already
    const int v = (int)(0xffffffffu - (unsigned)(key & 0xffffffffu));
    LA_TRY(search(v, M->L));
    min_update_kernel<<<vgrid(n), 256>>>(n, M->dist.as<int>() + (size_t)M->L * n,
                                         M->mind.as<int>());
    LA_CUDA_TRY(cudaGetLastError());
    M->L++;
  }
  const int L = M->L, np = L * (L - 1) / 2;
  if (np == 0)
    return LA_OK;
  DevBuf masks, lohi;
  LA_TRY(masks.alloc(sizeof(unsigned) * 2));
  LA_TRY(lohi.alloc(sizeof(int) * 2 * 28));
  LA_CUDA_TRY(cudaMemset(masks.p, 0, sizeof(unsigned) * 2));
  std::vector<int> init(56);
  for (int p = 0; p < 28; p++) {
    init[p] = INT_MAX;
    init[28 + p] = INT_MIN;
  }
  LA_CUDA_TRY(cudaMemcpy(lohi.p, init.data(), sizeof(int) * 56, cudaMemcpyHostToDevice));
  pair_sign_kernel<<<vgrid(n), 256>>>(n, L, M->tai.as<int>(), M->taj.as<int>(),
                                      M->dist.as<int>(), masks.as<unsigned>());
  pair_range_kernel<<<vgrid(n), 256>>>(n, L, M->dist.as<int>(), lohi.as<int>(),
                                       lohi.as<int>() + 28);
  LA_CUDA_TRY(cudaGetLastError());
  unsigned mk[2];
  int lh[56];
  LA_CUDA_TRY(cudaMemcpy(mk, masks.p, sizeof(mk), cudaMemcpyDeviceToHost));
  LA_CUDA_TRY(cudaMemcpy(lh, lohi.p, sizeof(lh), cudaMemcpyDeviceToHost));
  int p = 0;
  for (int a = 0; a < L; a++)
    for (int b = a + 1; b < L; b++, p++) {
      const bool pos = (mk[0] >> p) & 1u, neg = (mk[1] >> p) & 1u;
      if (pos == neg)
        continue; // not monotone, or constant along every entry
      cands.push_back({a, b, pos ? 1 : -1, (long long)lh[28 + p] - lh[p]});
    }
  return LA_OK;
}

la_status landmarks_device_coordinate(LandmarksDevice *M, const PartitionCand &c, int *f) {
  const int n = M->n;
  if (!M->f.p)
    LA_TRY(M->f.alloc(sizeof(int) * n));
  coordinate_kernel<<<vgrid(n), 256>>>(n, M->dist.as<int>() + (size_t)c.a * n,
                                       M->dist.as<int>() + (size_t)c.b * n, c.sign,
                                       M->f.as<int>());
  LA_CUDA_TRY(cudaGetLastError());
  LA_CUDA_TRY(cudaMemcpy(f, M->f.p, sizeof(int) * n, cudaMemcpyDeviceToHost));
  return LA_OK;
}

// One component (members ascending, more than two nodes): its Cuthill-McKee
// order, node + base, into out[0, size).
la_status rcm_device_component(RcmDevice *D, const int *members, int size, int *out) {
  DevBuf mem;
  LA_TRY(mem.upload(members, sizeof(int) * size));
  int src = -1, reached = 0, height = 0;
  LA_TRY(D->argmin(mem.as<int>(), size, &src));
  std::vector<int> ls;
  for (;;) { // PseudoDiameter
    LA_TRY(D->bfs(src, reached, ls, &height));
    const int last0 = ls[height - 1], last_m = ls[height] - last0;
    int first = -1;
    for (int chosen = 0; chosen < 5; chosen++) {
      int sel = -1;
      LA_TRY(D->argmin(D->queue.as<int>() + last0, last_m, &sel));
      if (sel < 0)
        break;
      if (first < 0)
        first = sel;
      mark_kernel<<<1, kThreads, 0, D->st>>>(sel, D->deg.as<int>(), D->ai.as<int>(),
                                            D->aj.as<int>(), D->base);
      LA_CUDA_TRY(cudaGetLastError());
    }
    if (first < 0)
      break;
    int h2 = 0;
    LA_TRY(D->bfs(first, reached, ls, &h2));
    if (h2 <= height)
      break;
    src = first;
  }
  // Cuthill-McKee sweep from src
  LA_TRY(D->bfs(src, reached, ls, &height));
  if (ls[height] != size) {
    set_error("RCM: a component's search reached %d of its %d nodes", ls[height], size);
    return LA_ERR_INVALID_ARG;
  }
  LA_TRY(D->sweep(src, height));
  DevBuf o;
  LA_TRY(o.alloc(sizeof(int) * size));
  add_base_copy_kernel<<<blocks_for(size), kThreads, 0, D->st>>>(size, D->cm.as<int>(), D->base,
                                                                  o.as<int>());
  LA_CUDA_TRY(cudaGetLastError());
  LA_CUDA_TRY(cudaMemcpy(out, o.p, sizeof(int) * size, cudaMemcpyDeviceToHost));
  // leave the level array clear for the next component
  bfs_reset_kernel<<<blocks_for(reached), kThreads, 0, D->st>>>(reached, D->queue.as<int>(),
                                                                D->level.as<int>());
  LA_CUDA_TRY(cudaGetLastError());
  LA_CUDA_TRY(cudaStreamSynchronize(D->st));
  return LA_OK;
}

} // namespace la

namespace la {
namespace {

// pattern check on the device: columns in range, rows non-decreasing, and
// every entry (j, i) stored as often in row j as (i, j) is in row i -- the
// condition the host's transpose comparison tests.  flag = 1 if it fails.
__global__ void symmetric_check_kernel(const int n, const int base, const int *__restrict__ ai,
                                       const int *__restrict__ aj, int *flag) {
  bool bad = false;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int a = __ldg(ai + i) - base, e = __ldg(ai + i + 1) - base;
    for (int k = a; k < e && !bad; k++) {
      const int j = __ldg(aj + k) - base;
      if (j < 0 || j >= n || (k > a && __ldg(aj + k - 1) > __ldg(aj + k))) {
        bad = true;
        break;
      }
      if (k > a && __ldg(aj + k - 1) == __ldg(aj + k))
        continue; // a run of equal entries is counted at its first
      int run = 1;
      while (k + run < e && __ldg(aj + k + run) == __ldg(aj + k))
        run++;
      // count i in row j (non-decreasing: lower / upper bound)
      int lo = __ldg(ai + j) - base, hi = __ldg(ai + j + 1) - base;
      int l = lo, h = hi;
      while (l < h) {
        const int m = (l + h) >> 1;
        if (__ldg(aj + m) - base < i)
          l = m + 1;
        else
          h = m;
      }
      int u = l;
      while (u < hi && __ldg(aj + u) - base == i)
        u++;
      if (u - l != run)
        bad = true;
    }
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0)
    *flag = 1;
}

} // namespace

// la_rcm_device's front: the pattern check on the device and, for a
// connected pattern that qualifies, the whole ordering there (*handled);
// otherwise the caller runs rcm() (host components, large ones on the
// device).
la_status rcm_device_connected(int n, int base, const int *ai, const int *aj, int *iperm,
                               int *perm, bool *handled) {
  *handled = false;
  std::vector<int> deg(n);
  int maxdeg = 0;
  for (int i = 0; i < n; i++) {
    deg[i] = ai[i + 1] - ai[i];
    maxdeg = std::max(maxdeg, deg[i]);
  }
  la_status st = LA_OK;
  RcmDevice *D = rcm_device_create(n, base, ai, aj, deg.data(), &st);
  if (!D)
    return st;
  struct Owner {
    RcmDevice *d;
    ~Owner() { rcm_device_destroy(d); }
  } own{D};
  LA_CUDA_TRY(cudaMemset(D->count.p, 0, sizeof(int)));
  symmetric_check_kernel<<<blocks_for(n), kThreads>>>(n, base, D->ai.as<int>(), D->aj.as<int>(),
                                                      D->count.as<int>());
  LA_CUDA_TRY(cudaGetLastError());
  int bad = 0;
  LA_CUDA_TRY(cudaMemcpy(&bad, D->count.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (bad) {
    set_error("la_rcm_device needs a structurally symmetric pattern");
    return LA_ERR_INVALID_ARG;
  }
  if (n < kRcmDeviceMin || maxdeg > kRcmMaxDegree)
    return LA_OK; // the caller's path
  // connected?  one device BFS from node 0
  std::vector<int> ls;
  int reached = 0, height = 0;
  LA_TRY(D->bfs(0, reached, ls, &height));
  const int all = reached;
  bfs_reset_kernel<<<blocks_for(reached), kThreads>>>(reached, D->queue.as<int>(),
                                                       D->level.as<int>());
  LA_CUDA_TRY(cudaGetLastError());
  if (all != n)
    return LA_OK; // several components: the caller's path
  // one component, members 0 .. n-1 ascending
  std::vector<int> members(n);
  for (int i = 0; i < n; i++)
    members[i] = i;
  LA_TRY(rcm_device_component(D, members.data(), n, iperm));
  std::reverse(iperm, iperm + n);
  for (int i = 0; i < n; i++)
    perm[iperm[i] - base] = i + base;
  *handled = true;
  return LA_OK;
}

} // namespace la
