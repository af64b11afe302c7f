"""Calibration sweeps over several GPUs: whole simulations are split across
ranks largest first (fundem_b200.batch.shard) and each rank's results are
gathered on every rank (run_sharded).  On CPU: the split itself, and the
orchestration over gloo with world size 2, each rank stepping a stand-in
batch (the simulations exchange nothing while they run, so the stand-in
exercises everything but the device)."""
import os
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_shard_splits_whole_simulations_evenly():
    from fundem_b200 import batch
    _, params = batch.calibration_scenarios(n_sims=256, seed=1)
    costs = np.array([p["n"] for p in params], float) * 20000
    for world in (1, 2, 4, 8):
        parts = batch.shard(costs, world)
        assert len(parts) == world
        assert sorted(i for p in parts for i in p) == list(range(256))
        load = np.array([costs[p].sum() for p in parts])
        # largest-first assignment: no rank exceeds another by more than one simulation
        assert load.max() - load.min() <= costs.max()
        assert parts == batch.shard(costs, world)           # every rank computes the same split
    assert batch.shard([5.0, 1.0, 1.0], 2) == [[0], [1, 2]]
    assert batch.shard([], 3) == [[], [], []]


class _Sim:
    def __init__(self, sc):
        self.pos = np.array(sc.particles.pos, float)

    def state(self):
        return {"pos": self.pos}


class _Batch:
    """Stands in for batch.Batch on the CPU: every step lowers each particle
    by 1 micrometre."""

    def __init__(self, scenarios, device=0):
        self.sims = [_Sim(sc) for sc in scenarios]

    def run_graphs(self, steps, chunk):
        for s in self.sims:
            s.pos = s.pos - np.array([0.0, 0.0, 1e-6 * steps])

    def close(self):
        self.sims = []


def _rank(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from fundem_b200 import batch
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        scs, _ = batch.calibration_scenarios(n_sims=40, seed=3)
        res = batch.run_sharded(scs, 50, 25, rank, world, dist=dist, batch_cls=_Batch)
        out[rank] = res
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_run_sharded_two_ranks():
    port = 29600 + os.getpid() % 1000
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    sys.path.insert(0, ROOT)
    from fundem_b200 import batch
    scs, _ = batch.calibration_scenarios(n_sims=40, seed=3)
    want = {i: float(sc.particles.pos[:, 2].mean() - 50e-6) for i, sc in enumerate(scs)}
    for r in (0, 1):
        assert sorted(res[r]) == list(range(40))
        assert all(res[r][i] == pytest.approx(want[i], rel=0, abs=1e-15) for i in range(40))
    assert res[0] == res[1]


class _FailingBatch(_Batch):
    """A stand-in whose construction fails on rank 1 (a simulation that
    cannot be built there)."""

    def __init__(self, scenarios, device=0):
        import torch.distributed as dist
        if dist.get_rank() == 1:
            raise ValueError("no room for the batch")
        super().__init__(scenarios, device)


def _rank_failing(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from fundem_b200 import batch
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        scs, _ = batch.calibration_scenarios(n_sims=12, seed=3)
        try:
            batch.run_sharded(scs, 10, 5, rank, world, dist=dist, batch_cls=_FailingBatch)
            out[rank] = "returned"
        except RuntimeError as exc:
            out[rank] = str(exc)
    finally:
        dist.destroy_process_group()


def test_run_sharded_failure_reaches_every_rank():
    """A rank whose batch fails still joins the gather; every rank then raises
    the same error instead of waiting for the process-group timeout."""
    port = 29700 + os.getpid() % 1000
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_failing, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    for r in (0, 1):
        assert "rank 1: ValueError: no room for the batch" in res[r]


class _Tiled:
    """Stands in for batch.TiledBatch on the CPU: every step lowers each
    particle by 1 micrometre."""

    def __init__(self, scenarios, device=0):
        self.pos = [np.array(sc.particles.pos, float) for sc in scenarios]

    def run(self, steps):
        self.pos = [p - np.array([0.0, 0.0, 1e-6 * steps]) for p in self.pos]

    def states(self):
        return [{"pos": p} for p in self.pos]

    def close(self):
        self.pos = []


def _rank_tiled(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from fundem_b200 import batch
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        scs, _ = batch.calibration_scenarios(n_sims=40, seed=3)

        def timer():
            return lambda: 0.25 + rank       # seconds of this rank's timed steps
        res, secs, parts = batch.run_sharded_tiled(scs, 50, rank, world, dist=dist, warmup=10, timer=timer,
                                                   tiled_cls=_Tiled)
        out[rank] = (res, secs, parts)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_run_sharded_tiled_two_ranks():
    """Each rank tiles its share into one stand-in simulation; every rank
    ends with every simulation's result, the split, and both ranks'
    timings (the bench takes the maximum)."""
    port = 29800 + os.getpid() % 1000
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_tiled, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    sys.path.insert(0, ROOT)
    from fundem_b200 import batch
    scs, _ = batch.calibration_scenarios(n_sims=40, seed=3)
    want = {i: float(sc.particles.pos[:, 2].mean() - 60e-6) for i, sc in enumerate(scs)}
    parts = batch.shard([len(sc.particles) * 50 for sc in scs], 2)
    for r in (0, 1):
        got, secs, p = res[r]
        assert sorted(got) == list(range(40))
        assert all(got[i] == pytest.approx(want[i], rel=0, abs=1e-15) for i in range(40))
        assert secs == [0.25, 1.25] and p == parts
    assert res[0] == res[1]
