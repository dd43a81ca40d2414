"""The bench's N > 1 path on CPU: two gloo ranks.  Each rank solves its own
problem (distinct seeds); the job's time is the slowest rank's and its value
sums every rank's evaluations over that time."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import sys
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        ms = bench.allmax(10.0 + 5.0 * rank, world)
        q.put((rank, bench.rank_seed(2, rank), ms, bench.job_value(1.0e9, ms, world)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(world))
    seeds = {g[1] for g in got}
    assert len(seeds) == world  # independent problems
    for _, _, ms, value in got:
        assert ms == pytest.approx(15.0)
        assert value == pytest.approx(2 * 1.0e9 / 0.015)
