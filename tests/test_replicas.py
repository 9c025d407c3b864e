"""Replica timing of bench.py under torch.distributed, on CPU with gloo.

bench.py runs one independent replica per GPU; the only collective is the
max-over-ranks reduction of each rank's timed region.  These tests run that
reduction in two gloo ranks and check the whole-job aggregate."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        t = [12.5, 20.0][rank]                     # per-rank device ms of the timed region
        t_max = bench.max_over_ranks(t, dist, "cpu")
        e2e = bench.max_over_ranks([0.3, 0.1][rank], dist, "cpu")
        q.put((rank, t_max, e2e, bench.aggregate_mcells(128 ** 3, 10, world, t_max)))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t_max, e2e, value in out:
        assert t_max == 20.0 and e2e == 0.3
        assert value == pytest.approx(128 ** 3 * 10 * 2 / 0.020 / 1e6)


def test_single_rank_needs_no_process_group():
    import bench
    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5
    assert bench.aggregate_mcells(64 ** 3, 100, 1, 1000.0) == pytest.approx(64 ** 3 * 100 / 1e6)
