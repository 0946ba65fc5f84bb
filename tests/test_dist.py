"""Sharding the SpMV over ranks (linearalgebra_b200.dist) on CPU.

* the row blocks equal the reference's own LoadPrefixBalancedPartitionPos
  (utils/utils.h:187-222) as ParallelSPMV calls it, through the compiled
  reference;
* two gloo ranks: each builds its block of rows, the x slices are
  all-gathered, every rank multiplies its block (here with the oracle's
  serial SpMV, the reference's row order) and the gathered result equals the
  whole-matrix product bit for bit."""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

from linearalgebra_b200 import dist, gen

ROOT = Path(__file__).resolve().parent.parent


def _ragged(n, seed):
    r = np.random.default_rng(seed)
    lens = r.integers(0, 6, n)
    lens[r.random(n) < 0.02] = min(200, n)  # a few long rows
    lens[: n // 10] = 0                      # a run of empty rows
    ai = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    aj = np.concatenate([np.sort(r.choice(n, k, replace=False)) if k else np.zeros(0, int)
                         for k in lens]).astype(np.int32)
    return n, ai, aj, r.standard_normal(int(ai[-1]))


def test_row_blocks_match_reference_partition(orc):
    rf = orc.ref()
    if rf is None:
        pytest.skip("compiled reference not available")
    P = orc.ptr
    mats = [gen.laplacian_2d(40), gen.powerlaw(20_000, seed=3), _ragged(5_000, 1), _ragged(7, 2)]
    for n, ai, aj, av in mats:
        for nparts in (1, 2, 3, 4, 7, 8, 13):
            ours = dist.row_blocks_by_nnz(ai, nparts)
            ref = np.zeros(nparts + 1, np.int32)
            rf.la_ref_prefix_partition(n, P(np.ascontiguousarray(ai, np.int32)), nparts, P(ref))
            assert np.array_equal(ours, ref), (n, nparts, ours, ref)
            assert ours[0] == 0 and ours[-1] == n and np.all(np.diff(ours) >= 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch
    import torch.distributed as tdist
    sys.path.insert(0, str(ROOT))
    import oracle
    from linearalgebra_b200 import dist as d, gen as g
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    tdist.init_process_group("gloo", rank=rank, world_size=world)
    n, ai, aj, av = g.powerlaw(30_000, seed=5)
    x = g.uniform_vector(n, 1)
    start = d.row_blocks_by_nnz(ai, world)
    r0, r1 = int(start[rank]), int(start[rank + 1])
    bai, baj, bav = d.block_rows(ai, aj, av, r0, r1)
    # every rank owns its slice of x; the exchange gathers them all
    cap = int(np.max(np.diff(start)))
    mine = torch.zeros(cap, dtype=torch.float64)
    mine[: r1 - r0] = torch.as_tensor(x[r0:r1])
    full = torch.empty(cap * world, dtype=torch.float64)
    tdist.all_gather_into_tensor(full, mine)
    xg = np.concatenate([full[i * cap: i * cap + int(start[i + 1] - start[i])].numpy()
                         for i in range(world)])
    y = np.zeros(r1 - r0)
    P = oracle.ptr
    oracle.port().oracle_serial_spmv(r1 - r0, 0, P(bai), P(baj), P(bav), P(xg), P(y), 1.0, 0.0)
    ys = torch.zeros(cap, dtype=torch.float64)
    ys[: r1 - r0] = torch.as_tensor(y)
    yall = torch.empty(cap * world, dtype=torch.float64)
    tdist.all_gather_into_tensor(yall, ys)
    yg = np.concatenate([yall[i * cap: i * cap + int(start[i + 1] - start[i])].numpy()
                         for i in range(world)])
    ref = np.zeros(n)
    oracle.port().oracle_serial_spmv(n, 0, P(ai), P(aj), P(av), P(x), P(ref), 1.0, 0.0)
    tdist.barrier()
    tdist.destroy_process_group()
    out.put((rank, bool(np.array_equal(xg, x)), bool(np.array_equal(yg, ref))))


def test_two_rank_block_spmv_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got == [(0, True, True), (1, True, True)]


# ------------------------------------------------------------ DistSPMV
class _CpuPlan:
    """Stand-in for the block's SpMV kernel only: gathers x from the slices it
    is given (this rank's and its peers' memory) and multiplies the block with
    the oracle's serial SpMV (the reference's row order)."""

    def __init__(self, rows, base, bai, baj, bav, slow):
        self.rows, self.base = rows, base
        self.bai, self.baj, self.bav = bai, baj, bav
        self.slow = slow

    def xparts(self, slices, starts, y, alpha, beta):
        import time
        import oracle
        if self.slow:  # a late reader: its peers finish and move on first
            time.sleep(0.3)
        x = np.concatenate([np.asarray(s)[: int(starts[r + 1] - starts[r])]
                            for r, s in enumerate(slices)])
        yn = y.numpy()
        P = oracle.ptr
        oracle.port().oracle_serial_spmv(self.rows, self.base, P(self.bai), P(self.baj),
                                         P(self.bav), P(x), P(yn), float(alpha), float(beta))
        return y


class _CpuBackend:
    """DistSPMV's device side on the host: the plan above, CPU tensors, and
    the symmetric slices as files mapped by every rank (peer memory), with
    the gloo barrier standing in for the device-side one."""

    def __init__(self, folder, slow):
        self.folder, self.slow = folder, slow

    def plan(self, rows, ncols, base, bai, baj, bav, kind):
        return _CpuPlan(rows, base, bai, baj, bav, self.slow)

    def empty(self, size):
        import torch
        return torch.empty(size, dtype=torch.float64)

    def zeros(self, size):
        import torch
        return torch.zeros(size, dtype=torch.float64)

    def symmetric(self, cap, group):
        import torch
        import torch.distributed as tdist
        rank, world = tdist.get_rank(group), tdist.get_world_size(group)
        mine = np.memmap(Path(self.folder) / f"slice{rank}", np.float64, "w+", shape=(cap,))
        tdist.barrier(group)
        peers = [mine if r == rank else
                 np.memmap(Path(self.folder) / f"slice{r}", np.float64, "r+", shape=(cap,))
                 for r in range(world)]
        return torch.from_numpy(mine), peers, lambda: tdist.barrier(group)


def _dist_rank(rank, world, port, folder, out):
    import torch
    import torch.distributed as tdist
    sys.path.insert(0, str(ROOT))
    import oracle
    from linearalgebra_b200 import dist as d, gen as g
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    tdist.init_process_group("gloo", rank=rank, world_size=world)
    n, ai, aj, av = g.powerlaw(30_000, seed=7)
    x0 = g.uniform_vector(n, 2)
    y0 = g.uniform_vector(n, 3)
    P = oracle.ptr
    results = {}
    for mode in ("slices", "allgather"):
        sub = Path(folder) / mode
        sub.mkdir(exist_ok=True)
        ds = d.DistSPMV(None, n, ai, aj, av, mode=mode,
                        backend=_CpuBackend(sub, slow=(rank == world - 1)))
        r0, r1 = ds.rows
        ds.x_slice[:] = torch.as_tensor(x0[r0:r1])
        y = torch.as_tensor(y0[r0:r1].copy())
        want_x, want_y = x0.copy(), y0.copy()
        ok = True
        for _ in range(3):  # y fed back as x: each step rewrites the slices
            ds(y, 0.5, 0.25)
            ds.x_slice[:] = y
            oracle.port().oracle_serial_spmv(n, 0, P(ai), P(aj), P(av), P(want_x), P(want_y),
                                             0.5, 0.25)
            want_x = want_y.copy()
            ok &= bool(np.array_equal(y.numpy(), want_y[r0:r1]))
        results[mode] = ok
    tdist.barrier()
    tdist.destroy_process_group()
    out.put((rank, results["slices"], results["allgather"]))


def test_two_rank_dist_spmv_iterates_gloo(tmp_path):
    """DistSPMV itself on two gloo ranks, both modes, y fed back as x for three
    steps: every rank's block equals the whole-matrix iteration bit for bit.
    The last rank reads its peers' slices late, so a rank that rewrote its
    slice before every peer had read it would show up as a mismatch."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_dist_rank, args=(r, 2, port, str(tmp_path), q))
             for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got == [(0, True, True), (1, True, True)]
