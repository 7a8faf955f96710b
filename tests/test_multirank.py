"""The replica path's whole-job reduction across ranks (bench.reduce_over_ranks): two gloo
ranks on the CPU, each with its own time and unit count."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime
    import sys
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms, units = bench.reduce_over_ranks(10.0 + 5.0 * rank, 1000 * (rank + 1), "cpu")
        q.put((rank, ms, units))
    finally:
        dist.destroy_process_group()


def test_reduce_over_two_gloo_ranks():
    ctx = torch.multiprocessing.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, ms, units in got:
        assert ms == 15.0        # the slower rank's time
        assert units == 3000.0   # both ranks' units


def test_single_rank_is_unchanged():
    import sys
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reduce_over_ranks(12.5, 7, "cpu") == (12.5, 7.0)
