"""Multi-rank host logic of bench.py on CPU with two gloo ranks (no GPU).

The LenseFlow path shards by independent maps, so ranks exchange nothing but
the barrier and the max-over-ranks timing reduction; this checks that both
ranks agree on the slowest rank's time and on the whole-job throughput.
"""
import datetime
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    dist.barrier()
    ms = bench.max_over_ranks(10.0 + 5.0 * rank, dist, "cpu")
    q.put((rank, ms, bench.aggregate_value(world, 64, 5, ms)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_the_slowest_rank():
    import multiprocessing as mp
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
    assert [r[1] for r in res] == [15.0, 15.0]
    assert all(abs(r[2] - 2 * 64 * 5 / 0.015) < 1e-6 for r in res)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(12.5) == 12.5
    assert bench.aggregate_value(1, 64, 10, 100.0) == pytest.approx(6400.0)
