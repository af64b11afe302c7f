"""Sector periodicity (LSSolver::addPeriodicBoundarySector,
PeriodicBoundary.h:319-425) on the GPU, against the CPU oracle and against
the reference's own build (tests/golden/sector.npz).

The turned images come from sines, cosines and square roots: the GPU path
calls CUDA's, the oracle the host library's, so image positions may differ in
the last bit between the two.  Pair lists are compared exactly; overlaps of
the image lists to 1e-9 relative and states to the tolerances of the other
parity tests.  Against the reference build, which calls the same CUDA
functions, the image lists' overlaps are compared bit for bit."""
import numpy as np
import pytest

from conftest import canonical, golden_contacts, golden_state, keys, load_golden, rel_err, scenario_sha
import parity_cases as PC

pytestmark = pytest.mark.gpu

KINDS = ("pp", "pw", "gx", "gy", "gxy", "gr90", "gr180", "gr270")
SECTOR = (5, 6, 7)


def _pair(fundem, oracle_mod):
    sc = PC.sector()
    return sc, fundem.Simulation.from_scenario(sc), oracle_mod.OracleWorld.from_scenario(sc)


def _same(got, ref, bitwise):
    got, ref = canonical(got), canonical(ref)
    assert np.array_equal(keys(got), keys(ref))
    if len(ref["overlap"]):
        if bitwise:
            assert np.array_equal(got["overlap"], ref["overlap"])
        else:
            assert rel_err(got["overlap"], ref["overlap"]) < 1e-9
        assert np.abs(got["normal"] - ref["normal"]).max() < 1e-12
        assert np.abs(got["point"] - ref["point"]).max() < 1e-12 * max(1.0, np.abs(ref["point"]).max())


def test_sector_initial_detection_vs_oracle(fundem, oracle_mod):
    sc, g, o = _pair(fundem, oracle_mod)
    g.detect()
    o.initial_detect()
    for k in range(8):
        _same(g.contacts(k), o.contacts(k), bitwise=k not in SECTOR)
    # every image set meets bodies in this case
    for k in SECTOR:
        assert len(o.contacts(k)["master"]) > 0, k
    g.sync()


def test_sector_steps_vs_oracle(fundem, oracle_mod):
    """Twelve steps: the body that starts outside the x face is turned back
    into the sector on the first, and every list, force and state agrees."""
    sc, g, o = _pair(fundem, oracle_mod)
    g.detect()
    o.initial_detect()
    for s in range(12):
        g.step(1)
        o.step(1)
        for k in range(8):
            _same(g.contacts(k), o.contacts(k), bitwise=False)
        sg, so = g.state(), o.state()
        assert rel_err(sg["force"], so["force"]) < 1e-10
        assert rel_err(sg["torque"], so["torque"]) < 1e-10
        assert rel_err(sg["pos"], so["pos"]) < 1e-13
        assert rel_err(sg["vel"], so["vel"]) < 1e-10
        assert rel_err(sg["angvel"], so["angvel"]) < 1e-10
        assert rel_err(sg["quat"], so["quat"]) < 1e-13
    st = g.state()
    assert st["pos"][0, 0] > sc.domain_min[0]  # turned back in
    g.sync()


def _sim_at_reference(fundem, gold, step):
    g = fundem.Simulation.from_scenario(PC.sector())
    g.set_state(**golden_state(gold, step))
    g.set_state(wall=True, pos=gold[f"s{step}_wall_pos"], quat=gold[f"s{step}_wall_quat"])
    for ki, kind in enumerate(KINDS):
        c = golden_contacts(gold, step, kind)
        if len(c["master"]):
            g.set_contacts(ki, c["master"], c["slave"], c["spring"])
    return g


def test_sector_detection_vs_reference(fundem):
    """From the reference's dumped state at step s the detection gives its
    image lists, overlaps bit for bit."""
    gold = load_golden("sector")
    assert str(gold["scenario_sha256"]) == scenario_sha("sector")
    steps = [int(s) for s in gold["steps"]]
    n = 0
    for s in steps:
        if s - 1 not in steps:
            continue
        g = _sim_at_reference(fundem, gold, s - 1)
        g.set_state(**golden_state(gold, s))
        g.set_state(wall=True, pos=gold[f"s{s}_wall_pos"], quat=gold[f"s{s}_wall_quat"])
        g.detect()
        # the reference detects particle and wall pairs before the sector
        # wrap of that step; the dumped positions are after it
        for ki in SECTOR:
            ref = golden_contacts(gold, s, KINDS[ki])
            got = g.contacts(ki)
            assert np.array_equal(keys(canonical(got)), keys(canonical(ref))), (s, ki)
            if len(ref["overlap"]):
                assert np.array_equal(canonical(got)["overlap"], canonical(ref)["overlap"]), (s, ki)
        g.sync()
        n += 1
    assert n > 0


def test_sector_full_step_vs_reference(fundem):
    gold = load_golden("sector")
    steps = [int(s) for s in gold["steps"]]
    n = 0
    for s in steps:
        if s - 1 not in steps:
            continue
        g = _sim_at_reference(fundem, gold, s - 1)
        g.step_end()
        g.step_begin()
        st = g.state()
        ref = golden_state(gold, s)
        for ki, kind in enumerate(KINDS):
            r = golden_contacts(gold, s, kind)
            got = g.contacts(ki)
            assert np.array_equal(keys(canonical(got)), keys(canonical(r))), (s, kind)
            if len(r["spring"]):
                assert rel_err(canonical(got)["spring"], canonical(r)["spring"]) < 1e-8
        assert rel_err(st["pos"], ref["pos"]) < 1e-13
        assert rel_err(st["force"], ref["force"]) < 1e-10
        assert rel_err(st["torque"], ref["torque"]) < 1e-10
        g.sync()
        n += 1
    assert n > 0


def test_sector_trajectory_vs_reference(fundem):
    gold = load_golden("sector")
    g = fundem.Simulation.from_scenario(PC.sector())
    g.detect()
    done = 0
    for s in [int(x) for x in gold["steps"]]:
        g.step(s - done)
        done = s
        st = g.state()
        ref = golden_state(gold, s)
        assert rel_err(st["pos"], ref["pos"]) < 1e-10, s
        for ki, kind in enumerate(KINDS):
            assert np.array_equal(keys(canonical(g.contacts(ki))),
                                  keys(canonical(golden_contacts(gold, s, kind)))), (s, kind)
    g.sync()


def test_sector_neighbour_list_and_mixed(fundem):
    """With sector periodicity the neighbour list (forced on at this size)
    gives the cell search's steps bit for bit, bodies turned by the wrap
    included; the mixed-precision path follows FP64 closely."""
    def run(nl, precision):
        g = fundem.Simulation.from_scenario(PC.sector())
        g.set_neighbour_list(nl)
        g.set_precision(precision)
        g.detect()
        g.step(40)
        g.sync()
        st = g.state()
        c = g.contacts(0)
        g.close()
        return st, c
    cell, c_cell = run(0, fundem.FP64)
    nl, c_nl = run(1, fundem.FP64)
    assert np.array_equal(cell["pos"], nl["pos"]) and np.array_equal(cell["vel"], nl["vel"])
    assert np.array_equal(keys(canonical(c_cell)), keys(canonical(c_nl)))
    mixed, _ = run(0, fundem.FP32_MIXED)
    assert rel_err(mixed["pos"], cell["pos"]) < 1e-6
