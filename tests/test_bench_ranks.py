"""The multi-rank plumbing of bench.py on CPU: two gloo ranks, max-over-ranks timing and the whole-job
throughput (replicas: each rank evaluates its own copy of the workload)."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = bench.max_over_ranks(10.0 + 5.0 * rank)  # rank 1 is the slowest
        q.put((rank, ms, bench.aggregate_value(4_000_000, world, ms)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for rank, ms, value in res:
        assert ms == 15.0
        assert abs(value - 2 * 4_000_000 / 15e-3 / 1e6) < 1e-9
