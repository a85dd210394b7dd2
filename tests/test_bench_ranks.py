"""The multi-rank path of bench.py on CPU: two gloo ranks on 127.0.0.1 take the
slowest rank's time and report the whole-job rate (replicas, weak scaling)."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = 10.0 + 5.0 * rank  # rank 1 is the slow one
        m = bench.max_over_ranks(ms, world, device="cpu")
        e = bench.max_over_ranks(100.0 - rank, world, device="cpu")
        out[rank] = (m, e, bench.job_rate(1000, world, 4, m))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_take_the_slowest_time_and_the_whole_job_rate():
    ctx = mp.get_context("spawn")
    world, port = 2, _free_port()
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    assert res[0] == res[1]  # every rank sees the same reduced figures
    m, e, rate = res[0]
    assert m == 15.0 and e == 100.0
    assert rate == pytest.approx(1000 * 2 * 4 / 0.015)


def test_one_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(7.5, 1) == 7.5
    assert bench.job_rate(10, 1, 2, 1000.0) == pytest.approx(20.0)
