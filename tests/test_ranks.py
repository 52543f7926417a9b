"""The N > 1 path of bench.py on CPU: two gloo ranks, each timing its own
replica, reduce their timings to the maximum over ranks (every rank gets
it) and rank 0 turns it into the whole-job rate (replicas only: no other
collective is on the path)."""
import os
import socket
import sys

import pytest

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    # rank r took (100 + 50 r) ms for the headline and (300 - 100 r) ms for the e2e form
    ms = bench.max_over_ranks([100.0 + 50.0 * rank, 300.0 - 100.0 * rank], dist, "cpu")
    rate = bench.job_rate(world, 30, ms[0])
    out.put((rank, ms, rate))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_and_job_rate_with_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, rate in res:
        assert ms == [150.0, 300.0]  # the slowest rank's time for each form
        assert rate == pytest.approx(2 * 30 / 0.150)


def test_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks([1.5, 2.5]) == [1.5, 2.5]
    assert bench.job_rate(1, 30, 1500.0) == pytest.approx(20.0)

