"""The streams of a step.  After the hash stage the particle-wall list and,
with translated periodicity, the image lists run on streams of their own
beside the particle-particle list, with the bonds at the end of one of them;
with the per-stage timers on (fundem_set_profiling) every stage runs on the
simulation's stream in the reference's order (LSSolver.h:1201-1215 and
:780-784: particle pairs, walls, wraps, images).  The branches share nothing
they write, so both orders give the same run bit for bit, with plain
launches and in graph replays, periodic (bonds on the image branch) or not
(bonds on the wall branch)."""
import dataclasses

import numpy as np
import pytest

from conftest import canonical, keys

pytestmark = pytest.mark.gpu


def _slab(periodic):
    from fundem_b200 import workloads
    sim, sc, info = workloads.bonded_column(n=2048, footprint=(16, 16), seed=4, platen_speed=20.0)
    sim.close()
    if not periodic:
        sc = dataclasses.replace(sc, periodic_x=False, periodic_y=False)
    return sc


def _run(fundem, sc, serial, graph, steps=60, cache=-1):
    s = fundem.Simulation.from_scenario(sc, records=False)
    s.set_pair_cache(cache)
    s.set_profiling(serial)
    s.detect()
    if graph:
        for _ in range(steps // 20):
            s.step_graph(20)
    else:
        s.step(steps)
    s.sync()
    st = s.state()
    lists = {k: canonical(s.contacts(k)) for k in (fundem.PP, fundem.PW, fundem.GX, fundem.GY, fundem.GXY)}
    bonds = s.bonds()["activated"].copy()
    s.close()
    return st, lists, bonds


@pytest.mark.parametrize("periodic,cache", [(True, -1), (False, -1), (True, 1)])
def test_branches_match_the_serial_order(fundem, periodic, cache):
    """cache 1: the pair cache on at this size (slot filter, carried lists,
    the reverse index kept between rebuilds)."""
    sc = _slab(periodic)
    ref = _run(fundem, sc, serial=True, graph=False, cache=cache)
    assert sum(len(keys(c)) for c in ref[1].values()) > 1000
    for graph in (False, True):
        st, lists, bonds = _run(fundem, sc, serial=False, graph=graph, cache=cache)
        for k in ("pos", "vel", "angvel", "quat", "force", "torque"):
            assert np.array_equal(st[k], ref[0][k]), (graph, k)
        for kind, c in lists.items():
            assert np.array_equal(keys(c), keys(ref[1][kind])), (graph, kind)
            assert np.array_equal(c["spring"], ref[1][kind]["spring"]), (graph, kind)
        assert np.array_equal(bonds, ref[2]), graph


def test_fused_step_boundary_matches_the_hooked_steps(fundem):
    """fundem_step and its graph run one step's second half kick with the
    next step's first half kick and drift in one kernel (k_kick_drift); the
    hooked form (fundem_step_begin / fundem_step_end) launches them one by
    one.  Both give the same run bit for bit."""
    sc = _slab(True)
    runs = []
    for form in ("hooked", "step", "graph"):
        s = fundem.Simulation.from_scenario(sc, records=False)
        s.detect()
        if form == "hooked":
            for _ in range(40):
                s.step_begin()
                s.step_end()
        elif form == "step":
            s.step(40)
        else:
            s.step_graph(20)
            s.step_graph(20)
        s.sync()
        runs.append(s.state())
        s.close()
    for st in runs[1:]:
        for k in ("pos", "vel", "angvel", "quat", "force", "torque"):
            assert np.array_equal(st[k], runs[0][k]), k
