"""The bench's multi-rank (replica) path on CPU: two gloo ranks.

bench.py --gpus N runs N independent replicas (the solve does not shard);
the job time is the max over ranks of each rank's time and the value the
units all ranks processed over that time.  These are the helpers bench.py
uses for exactly that, exercised through a real two-process group."""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import pytest

torch = pytest.importorskip("torch")
ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mine = [0.25, 0.5][rank]              # each rank's own time
    t = bench.max_over_ranks(dist, mine, "cpu")
    v = bench.replica_value(world, 10, 1e9, t)
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, t, v))


def test_replicas_time_is_max_over_ranks_and_value_sums_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, v in got:
        assert t == 0.5                    # the slower rank's time, on every rank
        assert v == pytest.approx(2 * 10 * 1e9 / 0.5 / 1e9)  # 40 GB/s for the job


def test_single_rank_helpers():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.max_over_ranks(None, 0.3, "cpu") == 0.3
    assert bench.replica_value(1, 4, 2e9, 2.0) == pytest.approx(4.0)
