"""The replica harness of bench.py with two ranks on the CPU (gloo): every rank takes part in the
same collective, the job time is the slowest rank's, and only rank 0 reports.  The GPU runs use
the same helper over NCCL, one rank per GPU."""
from __future__ import annotations

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out):
    import datetime
    import sys
    from pathlib import Path

    sys.path.insert(0, str(Path(__file__).resolve().parent.parent))
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        r, w, local = bench._dist()
        ms = bench._max_over_ranks(1.5 + rank, dist, "cpu")  # rank 1 is the slower replica
        dist.barrier()
        out.put((r, w, local, ms))
    finally:
        dist.destroy_process_group()


def test_replicas_take_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert [(r, w, l) for r, w, l, _ in res] == [(0, 2, 0), (1, 2, 1)]
    assert all(ms == pytest.approx(2.5) for *_, ms in res)


def test_single_process_needs_no_group():
    import bench

    assert bench._max_over_ranks(3.25, None, "cpu") == 3.25
    assert torch.distributed.is_available()
