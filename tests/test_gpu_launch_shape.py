"""Launch shapes of the narrow phase (fundem_set_launch_shape) and their
autotuner.  The selection, predicate, contact-law and pair-sum kernels loop
over their work grid-stride and sum each pair's slots in a fixed order, so
every shape gives the same run bit for bit; only the speed changes."""
import numpy as np
import pytest

from conftest import canonical, keys

pytestmark = pytest.mark.gpu


def _slab(seed=3):
    from fundem_b200 import workloads
    sim, sc, info = workloads.bonded_column(n=2048, footprint=(16, 16), seed=seed)
    sim.close()
    return sc


def test_shapes_give_the_same_run(fundem):
    sc = _slab()
    out = []
    for shape in ((0, 0, 0, 0), (1, 1, 1, 1), (16, 12, 8, 2)):
        s = fundem.Simulation.from_scenario(sc, records=False)
        s.set_launch_shape(*shape)
        want = tuple(d if v == 0 else v for v, d in zip(shape, (4, 4, 4, 4)))
        assert s.launch_shape() == want
        s.detect()
        s.step(60)
        s.sync()
        out.append((s.state(), s.contacts(fundem.PP), s.contacts(fundem.GX)))
        s.close()
    for st, cpp, cgx in out[1:]:
        for k in ("pos", "vel", "force", "torque"):
            assert np.array_equal(st[k], out[0][0][k]), k
        assert np.array_equal(keys(canonical(cpp)), keys(canonical(out[0][1])))
        assert np.array_equal(keys(canonical(cgx)), keys(canonical(out[0][2])))


def test_shape_bounds(fundem):
    s = fundem.Simulation(device=0)
    with pytest.raises(fundem.FundemError):
        s.set_launch_shape(65, 0, 0, 0)
    with pytest.raises(fundem.FundemError):
        s.set_launch_shape(0, -1, 0, 0)
    s.close()


def test_autotuner_leaves_the_fastest_shape(fundem):
    from fundem_b200 import autotune
    sc = _slab(seed=5)
    s = fundem.Simulation.from_scenario(sc, records=False)
    s.detect()
    cands = ((0, 0, 0, 0), (8, 8, 8, 8), (2, 2, 2, 2))
    best, times = autotune.launch_shape(s, steps=10, candidates=cands)
    assert set(times) == set(cands) and best == min(times, key=times.get)
    assert s.launch_shape() == tuple(d if v == 0 else v for v, d in zip(best, (4, 4, 4, 4)))
    s.sync()
    s.close()


def test_autotuner_restart_runs_every_candidate_from_one_state(fundem):
    """restart=True: each candidate starts from one checkpoint, so the
    simulation ends `steps` steps after the state the tuner found, as an
    uninterrupted run does."""
    from fundem_b200 import autotune
    sc = _slab(seed=5)
    s = fundem.Simulation.from_scenario(sc, records=False)
    s.detect()
    s.step(20)
    cands = ((0, 0, 0, 0), (8, 2, 2, 8))
    best, times = autotune.launch_shape(s, steps=15, candidates=cands, restart=True)
    assert set(times) == set(cands) and best == min(times, key=times.get)
    s.sync()
    r = fundem.Simulation.from_scenario(sc, records=False)
    r.detect()
    r.step(35)
    r.sync()
    ss, sr = s.state(), r.state()
    for k in ("pos", "vel", "force", "torque"):
        assert np.array_equal(ss[k], sr[k]), k
    assert np.array_equal(keys(canonical(s.contacts(fundem.PP))), keys(canonical(r.contacts(fundem.PP))))
    s.close()
    r.close()
