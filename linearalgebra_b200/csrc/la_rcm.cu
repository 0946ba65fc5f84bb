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
// B200 design.  A level-synchronous BFS (one launch per level; a vertex is
// claimed by a compare-and-swap on its level, so the levels are the
// sequential search's) and packed (degree, index) minimum reductions give
// the source.  The sweep needs no sequential walk: a node of level l+1 is
// appended by the first node of level l, in the ordering, that neighbours
// it, so per level (1) every next-level node finds the smallest ordering
// position among its level-l neighbours (its parent), (2) every level-l
// node counts the next-level nodes it is the parent of, (3) a scan of the
// counts gives each parent's first slot, and (4) every parent sorts its
// children by (degree, index) into its slots.  Integer work only: the
// ordering equals the host's exactly.  Used for components of at least
// kRcmDeviceMin nodes whose rows hold at most kRcmMaxDegree entries (a
// parent's children are sorted in registers); the host orders the rest.
//
// Roofline: latency-bound (a few launches per BFS level); each level reads
// its nodes' rows once per step.

#include "la_device.cuh"
#include "la_internal.h"

#include <algorithm>
#include <climits>
#include <vector>

namespace la {
namespace {

constexpr int kThreads = 256;

// frontier [qs, qe) of queue, next level appended after qe
__global__ void bfs_expand_kernel(const int qs, const int qe, const int lev, int *queue,
                                  int *level, const int *__restrict__ ai,
                                  const int *__restrict__ aj, const int base, int *cnt) {
  for (int h = qs + blockIdx.x * blockDim.x + threadIdx.x; h < qe;
       h += gridDim.x * blockDim.x) {
    const int u = queue[h];
    for (int k = __ldg(ai + u) - base; k < __ldg(ai + u + 1) - base; k++) {
      const int v = __ldg(aj + k) - base;
      if (level[v] < 0 && atomicCAS(level + v, -1, lev) == -1)
        queue[qe + atomicAdd(cnt, 1)] = v;
    }
  }
}

// level[v] = -1 for the nodes a previous search reached
__global__ void bfs_reset_kernel(const int m, const int *queue, int *level) {
  for (int h = blockIdx.x * blockDim.x + threadIdx.x; h < m; h += gridDim.x * blockDim.x)
    level[queue[h]] = -1;
}

__global__ void bfs_start_kernel(const int src, int *queue, int *level) {
  queue[0] = src;
  level[src] = 0;
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

// (1) parent of each next-level node: smallest ordering position among its
// level-l neighbours
__global__ void parent_kernel(const int m, const int *nodes, const int lev, const int *level,
                              const int *pos, int *parent, const int *__restrict__ ai,
                              const int *__restrict__ aj, const int base) {
  for (int h = blockIdx.x * blockDim.x + threadIdx.x; h < m; h += gridDim.x * blockDim.x) {
    const int v = nodes[h];
    int p = INT_MAX;
    for (int k = __ldg(ai + v) - base; k < __ldg(ai + v + 1) - base; k++) {
      const int u = __ldg(aj + k) - base;
      if (level[u] == lev)
        p = min(p, pos[u]);
    }
    parent[v] = p;
  }
}

// (2) children per level-l position p in [p0, p0 + m)
__global__ void child_count_kernel(const int p0, const int m, const int *cm, const int lev,
                                   const int *level, const int *parent, int *cnt,
                                   const int *__restrict__ ai, const int *__restrict__ aj,
                                   const int base) {
  for (int h = blockIdx.x * blockDim.x + threadIdx.x; h < m; h += gridDim.x * blockDim.x) {
    const int p = p0 + h, u = cm[p];
    int c = 0;
    for (int k = __ldg(ai + u) - base; k < __ldg(ai + u + 1) - base; k++) {
      const int v = __ldg(aj + k) - base;
      c += level[v] == lev + 1 && parent[v] == p;
    }
    cnt[h] = c;
  }
}

// (3) exclusive scan of cnt[0, m) in place, one block walking 2048-entry
// chunks with a running carry
__global__ void __launch_bounds__(1024) scan_one_block_kernel(int *cnt, const int m) {
  __shared__ int wsum[32];
  __shared__ int carry;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0)
    carry = 0;
  __syncthreads();
  for (int c0 = 0; c0 < m; c0 += 2048) {
    const int i0 = c0 + 2 * tid;
    const int a = i0 < m ? cnt[i0] : 0, b = i0 + 1 < m ? cnt[i0 + 1] : 0;
    int incl = a + b;
    for (int k = 1; k < 32; k <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, incl, k);
      if (lane >= k)
        incl += t;
    }
    if (lane == 31)
      wsum[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      const int w = wsum[lane];
      int wi = w;
      for (int k = 1; k < 32; k <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, wi, k);
        if (lane >= k)
          wi += t;
      }
      wsum[lane] = wi - w;
    }
    __syncthreads();
    const int ex = carry + wsum[warp] + incl - (a + b);
    if (i0 < m)
      cnt[i0] = ex;
    if (i0 + 1 < m)
      cnt[i0 + 1] = ex + a;
    __syncthreads();
    if (tid == 1023)
      carry = ex + a + b;
    __syncthreads();
  }
}

// (4) each parent's children, sorted by (degree, node), into its slots
template <int MAXC>
__global__ void place_kernel(const int p0, const int m, const int q0, int *cm, int *pos,
                             const int lev, const int *level, const int *parent, const int *off,
                             const int *deg, const int *__restrict__ ai,
                             const int *__restrict__ aj, const int base) {
  for (int h = blockIdx.x * blockDim.x + threadIdx.x; h < m; h += gridDim.x * blockDim.x) {
    const int p = p0 + h, u = cm[p];
    int ch[MAXC];
    int c = 0;
    for (int k = __ldg(ai + u) - base; k < __ldg(ai + u + 1) - base && c < MAXC; k++) {
      const int v = __ldg(aj + k) - base;
      if (level[v] == lev + 1 && parent[v] == p) {
        int i = c++; // insertion by (degree, node)
        while (i > 0 && (deg[ch[i - 1]] > deg[v] || (deg[ch[i - 1]] == deg[v] && ch[i - 1] > v))) {
          ch[i] = ch[i - 1];
          i--;
        }
        ch[i] = v;
      }
    }
    const int o = q0 + off[h];
    for (int i = 0; i < c; i++) {
      cm[o + i] = ch[i];
      pos[ch[i]] = o + i;
    }
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
  int n = 0, base = 0;
  DevBuf ai, aj, deg, level, queue, pos, parent, cm, cnt, best, count;
  cudaStream_t st = nullptr;

  la_status init(int n_, int base_, const int *h_ai, const int *h_aj, const int *h_deg) {
    n = n_;
    base = base_;
    const int nnz = h_ai[n] - base;
    LA_TRY(ai.upload(h_ai, sizeof(int) * (n + 1)));
    LA_TRY(aj.upload(h_aj, sizeof(int) * std::max(nnz, 1)));
    LA_TRY(deg.upload(h_deg, sizeof(int) * n));
    for (DevBuf *b : {&level, &queue, &pos, &parent, &cm, &cnt})
      LA_TRY(b->alloc(sizeof(int) * n));
    LA_TRY(best.alloc(sizeof(unsigned long long)));
    LA_TRY(count.alloc(sizeof(int)));
    LA_CUDA_TRY(cudaMemset(level.p, 0xff, sizeof(int) * n));
    return LA_OK;
  }

  // BFS from src; lstart[l] = first queue slot of level l; returns levels.
  // The previous search's reached set (reached) is reset first.
  la_status bfs(int src, int &reached, std::vector<int> &lstart, int *height) {
    if (reached > 0) {
      bfs_reset_kernel<<<blocks_for(reached), kThreads, 0, st>>>(reached, queue.as<int>(),
                                                                 level.as<int>());
      LA_CUDA_TRY(cudaGetLastError());
    }
    bfs_start_kernel<<<1, 1, 0, st>>>(src, queue.as<int>(), level.as<int>());
    LA_CUDA_TRY(cudaGetLastError());
    lstart.assign(1, 0);
    int qs = 0, qe = 1;
    for (int lev = 1;; lev++) {
      lstart.push_back(qe);
      LA_CUDA_TRY(cudaMemsetAsync(count.p, 0, sizeof(int), st));
      bfs_expand_kernel<<<blocks_for(qe - qs), kThreads, 0, st>>>(
          qs, qe, lev, queue.as<int>(), level.as<int>(), ai.as<int>(), aj.as<int>(), base,
          count.as<int>());
      LA_CUDA_TRY(cudaGetLastError());
      int c = 0;
      LA_CUDA_TRY(cudaMemcpy(&c, count.p, sizeof(int), cudaMemcpyDeviceToHost));
      if (c == 0)
        break;
      qs = qe;
      qe += c;
    }
    reached = qe;
    *height = (int)lstart.size() - 1;
    return LA_OK;
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
  int *cm = D->cm.as<int>(), *pos = D->pos.as<int>();
  LA_CUDA_TRY(cudaMemcpyAsync(cm, &src, sizeof(int), cudaMemcpyHostToDevice, D->st));
  const int zero = 0;
  LA_CUDA_TRY(cudaMemcpyAsync(pos + src, &zero, sizeof(int), cudaMemcpyHostToDevice, D->st));
  for (int l = 0; l + 1 < height; l++) {
    const int p0 = ls[l], m = ls[l + 1] - ls[l];
    const int q0 = ls[l + 1], mq = ls[l + 2] - ls[l + 1];
    parent_kernel<<<blocks_for(mq), kThreads, 0, D->st>>>(
        mq, D->queue.as<int>() + q0, l, D->level.as<int>(), pos, D->parent.as<int>(),
        D->ai.as<int>(), D->aj.as<int>(), D->base);
    child_count_kernel<<<blocks_for(m), kThreads, 0, D->st>>>(
        p0, m, cm, l, D->level.as<int>(), D->parent.as<int>(), D->cnt.as<int>(),
        D->ai.as<int>(), D->aj.as<int>(), D->base);
    scan_one_block_kernel<<<1, 1024, 0, D->st>>>(D->cnt.as<int>(), m);
    place_kernel<kRcmMaxDegree><<<blocks_for(m), kThreads, 0, D->st>>>(
        p0, m, q0, cm, pos, l, D->level.as<int>(), D->parent.as<int>(), D->cnt.as<int>(),
        D->deg.as<int>(), D->ai.as<int>(), D->aj.as<int>(), D->base);
    LA_CUDA_TRY(cudaGetLastError());
  }
  DevBuf o;
  LA_TRY(o.alloc(sizeof(int) * size));
  add_base_copy_kernel<<<blocks_for(size), kThreads, 0, D->st>>>(size, cm, D->base, o.as<int>());
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
