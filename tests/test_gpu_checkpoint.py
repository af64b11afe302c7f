"""Checkpoint files: a run continued from a checkpoint repeats the
uninterrupted run bit for bit (state, contact history and bonds), and a file
for another setup is refused."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_restart_repeats_the_run(fundem, tmp_path):
    from fundem_b200 import workloads
    sim, sc, info = workloads.bonded_column(n=2048, footprint=(16, 16), seed=6)
    sim.close()
    a = fundem.Simulation.from_scenario(sc, records=False)
    a.detect()
    a.step(150)
    path = str(tmp_path / "mid.fdck")
    a.checkpoint_write(path)
    a.step(150)
    a.sync()
    b = fundem.Simulation.from_scenario(sc, records=False)
    b.checkpoint_read(path)
    b.step(150)
    b.sync()
    sa, sb = a.state(), b.state()
    for k in ("pos", "vel", "force"):
        assert np.array_equal(sa[k], sb[k]), k
    ca, cb = a.contacts(fundem.PP), b.contacts(fundem.PP)
    assert np.array_equal(ca["master"], cb["master"]) and np.array_equal(ca["spring"], cb["spring"])
    assert np.array_equal(a.bonds()["activated"], b.bonds()["activated"])
    # another setup: refused
    other, sc2, _ = workloads.bonded_column(n=1024, footprint=(16, 8), seed=6)
    with pytest.raises(fundem.FundemError):
        other.checkpoint_read(path)
    for s in (a, b, other):
        s.close()
