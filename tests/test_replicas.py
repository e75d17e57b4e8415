"""The multi-GPU replica bookkeeping of bench.py on CPU: two gloo processes stand in for two GPU
ranks.  Each rank times its own replica; every rank must see the slowest rank's time after the
reduction, and the job's rate counts every rank's units over that time."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import sys
    import datetime

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        r = bench.Replicas(dist, "cpu")
        r.barrier()
        mine = 10.0 * (rank + 1)           # this rank's timed region, ms
        slowest = r.max(mine)
        r.barrier()
        out[rank] = (mine, slowest, bench.Replicas.rate(1000.0, world, slowest / 1e3))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_max_over_ranks_and_rate(world):
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    slow = 10.0 * world
    for rank in range(world):
        mine, slowest, rate = res[rank]
        assert mine == 10.0 * (rank + 1)
        assert slowest == slow
        assert rate == pytest.approx(1000.0 * world / (slow / 1e3))


def test_single_process_needs_no_group():
    import sys

    sys.path.insert(0, ROOT)
    import bench

    r = bench.Replicas(None, "cpu")
    r.barrier()
    assert r.max(7.5) == 7.5
    assert bench.Replicas.rate(100.0, 1, 2.0) == 50.0
