"""Multi-rank host logic of bench.py on CPU: two gloo ranks (world size 2).

The path runs one independent replica per GPU; the only cross-rank steps are a
barrier and the MAX all-reduce of the timed durations, and only rank 0 prints.
No GPU: the ranks are CPU processes on 127.0.0.1.
"""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime
    import torch
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
    try:
        dist.barrier()
        ms = bench.max_over_ranks(1.5 + rank, dist, torch.device("cpu"))
        e2e = bench.max_over_ranks(10.0 - rank, dist, torch.device("cpu"))
        line = bench.rank_result({"value": 1, "ms": ms}, rank)
        q.put((rank, ms, e2e, line))
    finally:
        dist.destroy_process_group()


def test_two_ranks_agree_on_the_slowest_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get(timeout=5) for _ in range(2))
    for rank, ms, e2e, line in got:
        assert ms == 2.5 and e2e == 10.0
        assert (line is not None) == (rank == 0)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.max_over_ranks(3.0, None, None) == 3.0
    assert bench.rank_result({"a": 1}, 0) == '{"a": 1}' and bench.rank_result({"a": 1}, 1) is None
