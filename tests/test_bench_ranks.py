"""bench.py's multi-rank aggregation on CPU: two gloo ranks with different
times agree on the slowest one, and the job value counts every rank."""
import os
import sys
from pathlib import Path

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import bench
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    ms = bench.max_over_ranks(torch, 10.0 + 5.0 * rank, world, "cpu")
    q.put((rank, ms, bench.job_gbps(1e9, world, ms)))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_gloo():
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [15.0, 15.0]
    assert out[0][2] == pytest.approx(2 * 1e9 / 0.015 / 1e9)


def test_single_rank_passthrough():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.max_over_ranks(torch, 3.5, 1, "cpu") == 3.5
    assert bench.job_gbps(2e9, 1, 1000.0) == pytest.approx(2.0)
