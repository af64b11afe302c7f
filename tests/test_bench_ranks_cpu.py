"""bench.py's multi-rank aggregation over gloo on CPU, world size 2: every
rank reports the slowest rank's time, and the value counts all ranks'
particle steps."""
import os
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        ms = [2.0, 3.5][rank]  # per-rank timed region, ms
        t_max, value = bench.aggregate(ms, 1000, 10, world, dist, "cpu")
        out[rank] = (t_max, value)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_aggregate_two_ranks():
    port = 29500 + os.getpid() % 1000
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    for r in (0, 1):
        t_max, value = res[r]
        assert t_max == 3.5
        assert value == pytest.approx(2 * 1000 * 10 / 3.5e-3)


def test_aggregate_single():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.aggregate(4.0, 100, 5, 1, None, "cpu") == (4.0, 100 * 5 / 4e-3)
