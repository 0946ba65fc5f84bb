"""SpMV of one matrix sharded over the GPUs of a node.

The reference's ParallelSPMV splits the rows of A over threads by equal
nonzero shares, whole rows (LoadPrefixBalancedPartitionPos, utils/utils.h:
187-222, called from sparse_mat_op/spmv.hpp:31-57); here the same cut splits
them over ranks, one GPU each.  Rank r keeps the rows [start[r], start[r+1])
of A (global column indices) and the same slice of every vector, so an
iteration that feeds y back as x needs one exchange: every rank's SpMV reads
all of x.  Two ways to do it:

* ``mode="slices"``: x stays where it lives.  Each rank's slice is allocated
  in symmetric memory (torch.distributed._symmetric_memory), the peer
  addresses of all slices are exchanged once, and la_spmv_xparts reads every
  column from the slice that owns it, over NVLink for remote columns -- the
  exchange happens inside the SpMV kernel, no separate collective and no
  gathered copy.  A barrier across ranks orders the writers of x before the
  readers, and a second one after the SpMV orders the readers before the
  next write of any slice (an iteration that feeds y back as x would
  otherwise let a fast rank overwrite its slice while a peer still gathers
  from it).
* ``mode="allgather"``: the slices are all-gathered into one local buffer
  (NCCL) and the block reads them there -- the plain collective baseline.

Both compute, for every row, exactly the block SpMV of that row's rank.
"""
from __future__ import annotations

import numpy as np

from . import api


def row_blocks_by_nnz(ai, nparts: int) -> np.ndarray:
    """Row boundaries start[0..nparts] of the reference's partition: part t
    gets rows [start[t], start[t+1]), the t-th equal share of the nonzeros
    rounded to whole rows -- LoadPrefixBalancedPartitionPos(ai, ai + n, t,
    nparts) (utils/utils.h:187-222): lower_bound over ai[0..n) of the share's
    first nonzero (t*(w+1) for t < resid, else t*w + resid, with w = nnz //
    nparts and resid = nnz % nparts) plus ai[0]; part 0 starts at row 0 and
    the last part ends at row n."""
    ai = np.asarray(ai, dtype=np.int64)
    n = len(ai) - 1
    total = int(ai[n] - ai[0])
    w, resid = divmod(total, nparts)

    def share_start(t):
        return t * w + resid if t >= resid else t * (w + 1)

    start = np.empty(nparts + 1, dtype=np.int64)
    start[0] = 0
    for t in range(1, nparts):
        start[t] = np.searchsorted(ai[:n], share_start(t) + ai[0], side="left")
    start[nparts] = n
    return start


def block_rows(ai, aj, av, r0: int, r1: int):
    """CSR of rows [r0, r1) (global column indices kept; base preserved)."""
    ai = np.asarray(ai)
    base = int(ai[0])
    k0, k1 = int(ai[r0]) - base, int(ai[r1]) - base
    bai = (np.asarray(ai[r0:r1 + 1], dtype=np.int64) - int(ai[r0]) + base).astype(np.int32)
    return bai, np.ascontiguousarray(aj[k0:k1]), np.ascontiguousarray(av[k0:k1])


class CudaBackend:
    """The shipped device side of DistSPMV: the rank's block uploaded to its
    GPU and planned (la_spmv_plan_create), x slices in symmetric memory
    (torch.distributed._symmetric_memory) whose peer addresses la_spmv_xparts
    reads, and a barrier across the ranks ordered on the current stream."""

    def __init__(self):
        import torch
        self.torch = torch
        self.device = torch.device("cuda", torch.cuda.current_device())

    def plan(self, rows, ncols, base, bai, baj, bav, kind):
        return api.SPMV(api.CSR(rows, ncols, base, bai, baj, bav), kind)

    def empty(self, size):
        return self.torch.empty(size, dtype=self.torch.float64, device=self.device)

    def zeros(self, size):
        return self.torch.zeros(size, dtype=self.torch.float64, device=self.device)

    def symmetric(self, cap, group):
        """(this rank's buffer, every rank's buffer address, barrier)."""
        import torch.distributed._symmetric_memory as symm
        buf = symm.empty(cap, dtype=self.torch.float64, device=self.device)
        handle = symm.rendezvous(buf, group)
        return buf, [int(p) for p in handle.buffer_ptrs], handle.barrier


class DistSPMV:
    """y_r = alpha*A_r x + beta*y_r for this rank's block A_r of rows (see the
    module doc), FP64.

    group: an initialised torch.distributed process group over NCCL, one rank
    per GPU of the node, at most LA_SPMV_MAX_XPARTS ranks; every rank passes
    the same full CSR (host arrays) and keeps its block.  Write this rank's
    slice of x into ``x_slice``, then call on every rank; a call returns once
    every rank's SpMV has read x (in stream order), so ``x_slice`` may be
    rewritten right after it -- e.g. with y, to iterate.

    backend: the device side (plan, buffers, symmetric slices); CudaBackend
    unless a caller substitutes its own."""

    def __init__(self, group, n, ai, aj, av, kind=api.LA_SPMV_SEGSUM, mode="slices",
                 backend=None):
        import torch.distributed as dist
        self.group, self.mode = group, mode
        self.rank, self.world = dist.get_rank(group), dist.get_world_size(group)
        if self.world > api.LA_SPMV_MAX_XPARTS:
            raise ValueError(f"at most {api.LA_SPMV_MAX_XPARTS} ranks")
        if mode not in ("slices", "allgather"):
            raise ValueError("mode must be 'slices' or 'allgather'")
        self.backend = be = backend if backend is not None else CudaBackend()
        self.start = row_blocks_by_nnz(ai, self.world)
        r0, r1 = int(self.start[self.rank]), int(self.start[self.rank + 1])
        self.rows = (r0, r1)
        bai, baj, bav = block_rows(ai, aj, av, r0, r1)
        self.plan = be.plan(r1 - r0, n, int(np.asarray(ai)[0]), bai, baj, bav, kind)
        self._cap = max(int(np.max(np.diff(self.start))), 1)
        if mode == "slices":
            self._buf, self._ptrs, self._barrier = be.symmetric(self._cap, group)
            self.x_slice = self._buf[: r1 - r0]
        else:
            self._full = be.empty(self._cap * self.world)
            self._pad = be.zeros(self._cap)
            self.x_slice = self._pad[: r1 - r0]

    def __call__(self, y, alpha=1.0, beta=0.0):
        """y = alpha*A_r x + beta*y once every rank has written its x_slice."""
        import torch.distributed as dist
        if self.mode == "slices":
            self._barrier()  # every slice written before anyone reads
            self.plan.xparts(self._ptrs, self.start, y, alpha, beta)
            # every peer's SpMV has read this rank's slice before the caller
            # may rewrite it (write after read across GPUs)
            self._barrier()
            return y
        dist.all_gather_into_tensor(self._full, self._pad, group=self.group)
        parts = [self._full[i * self._cap:(i + 1) * self._cap] for i in range(self.world)]
        self.plan.xparts(parts, self.start, y, alpha, beta)
        return y
