"""Host logic of the launch-shape autotuner (fundem_b200.autotune) with a
stand-in simulation: the order of its calls, the timer, the choice, and the
temporary checkpoint of restart mode (written once, read before every
candidate, removed afterwards, also when a candidate fails)."""
import os

import pytest

from fundem_b200 import autotune


class FakeSim:
    """Records calls; a candidate's time is its first entry (seconds)."""

    def __init__(self, fail_on=None):
        self.calls = []
        self.shape = (0, 0, 0, 0)
        self.fail_on = fail_on
        self.written = None

    def set_launch_shape(self, *shape):
        self.shape = tuple(shape)
        self.calls.append(("shape", self.shape))

    def step(self, n):
        if self.fail_on is not None and self.shape == self.fail_on:
            raise RuntimeError("candidate failed")
        self.calls.append(("step", n))

    def sync(self):
        self.calls.append(("sync",))

    def checkpoint_write(self, path):
        assert os.path.exists(path)
        self.written = path
        self.calls.append(("write", path))

    def checkpoint_read(self, path):
        assert path == self.written and os.path.exists(path)
        self.calls.append(("read", path))


def _timer(sim):
    # the stop callable returns the running shape's first entry as seconds
    def start():
        return lambda: float(sim.shape[0])
    return start


def test_plain_mode_runs_candidates_one_after_another():
    sim = FakeSim()
    cands = ((3, 1, 1, 1), (1, 2, 2, 2), (2, 3, 3, 3))
    best, times = autotune.launch_shape(sim, steps=7, candidates=cands, timer=_timer(sim))
    assert best == (1, 2, 2, 2) and sim.shape == best
    assert times == {(3, 1, 1, 1): 3.0, (1, 2, 2, 2): 1.0, (2, 3, 3, 3): 2.0}
    # each candidate: shape, one untimed step, then the timed steps
    steps = [c[1] for c in sim.calls if c[0] == "step"]
    assert steps == [1, 7] * 3
    assert not any(c[0] in ("write", "read") for c in sim.calls)


def test_restart_mode_reads_one_checkpoint_before_every_candidate():
    sim = FakeSim()
    cands = ((2, 1, 1, 1), (1, 1, 1, 1))
    best, times = autotune.launch_shape(sim, steps=5, candidates=cands, timer=_timer(sim), restart=True)
    assert best == (1, 1, 1, 1) and sim.shape == best
    kinds = [c[0] for c in sim.calls]
    assert kinds.count("write") == 1 and kinds.count("read") == 2
    assert kinds[0] == "write"
    # no untimed step: every candidate starts from the checkpoint
    assert [c[1] for c in sim.calls if c[0] == "step"] == [5, 5]
    for i, c in enumerate(sim.calls):
        if c[0] == "read":
            assert sim.calls[i + 1][0] == "shape"
    assert not os.path.exists(sim.written)


def test_restart_mode_removes_its_checkpoint_when_a_candidate_fails():
    sim = FakeSim(fail_on=(4, 4, 4, 4))
    with pytest.raises(RuntimeError):
        autotune.launch_shape(sim, steps=3, candidates=((1, 1, 1, 1), (4, 4, 4, 4)), restart=True)
    assert sim.written is not None and not os.path.exists(sim.written)
