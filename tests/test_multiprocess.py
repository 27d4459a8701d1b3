"""The multi-GPU layout is replicas: each rank multiplies its own products, the
bench reports all ranks' products over the slowest rank's device time.  The
reduction logic runs here on CPU with two gloo ranks (no GPU, no NCCL)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime

    import torch.distributed as td
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    td.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
    try:
        import bench
        # rank r "measured" 10 + r milliseconds for 5 products
        ms = bench.max_over_ranks(10.0 + rank)
        value = bench.replica_throughput(world, 5, ms / 1000.0)
        q.put((rank, ms, value))
    finally:
        td.destroy_process_group()


def test_two_gloo_ranks_report_max_time_and_total_products():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(world))
    for rank, ms, value in got:
        assert ms == pytest.approx(11.0)          # the slower rank's time on every rank
        assert value == pytest.approx(2 * 5 / 0.011)  # both ranks' products over it


def test_single_process_is_identity():
    import bench
    assert bench.max_over_ranks(3.5) == 3.5
    assert bench.replica_throughput(1, 4, 2.0) == 2.0
