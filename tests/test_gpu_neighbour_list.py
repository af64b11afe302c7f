"""The particle-particle broad phase through the neighbour list gives the
same pairs as the cell search every step: bit-identical trajectories and
contact lists on a column that compresses (particles move, wrap across the
periodic seams), and the oracle's contacts on the parity cases."""
import numpy as np
import pytest

from conftest import canonical
import parity_cases as PC

pytestmark = pytest.mark.gpu


def test_neighbour_list_matches_cell_search(fundem):
    from fundem_b200 import workloads
    sim, sc, info = workloads.bonded_column(n=4096, footprint=(32, 16), seed=4, settle_steps=0)
    sim.close()
    runs = {}
    for mode in (0, 1):
        s = fundem.Simulation.from_scenario(sc, records=False)
        s.set_neighbour_list(mode)
        s.detect()
        s.step(600)
        s.sync()
        runs[mode] = (s.state(), s.contacts(fundem.PP), s.num_pairs(fundem.PP))
        s.close()
    (a, ca, pa), (b, cb, pb) = runs[0], runs[1]
    assert pa == pb
    assert np.array_equal(a["pos"], b["pos"]) and np.array_equal(a["force"], b["force"])
    assert np.array_equal(ca["master"], cb["master"]) and np.array_equal(ca["spring"], cb["spring"])


@pytest.mark.parametrize("name", ["cluster", "periodic"])
def test_neighbour_list_parity_cases(fundem, oracle_mod, name):
    sc = PC.CASES[name]()
    g = fundem.Simulation.from_scenario(sc)
    g.set_neighbour_list(1)
    o = oracle_mod.OracleWorld.from_scenario(sc)
    g.detect()
    o.initial_detect()
    for _ in range(5):
        g.step(1)
        o.step(1)
    for k in range(5):
        a, b = canonical(g.contacts(k)), canonical(o.contacts(k))
        assert np.array_equal(a["master"], b["master"]) and np.array_equal(a["slave"], b["slave"])
    g.close()
