"""The small pour at full size (1,000 superellipsoids from 4 templates, 32^3
grids, 642 nodes, six plane walls of a 20 x 20 x 40 mm box, seed 0) on the GPU
against the CPU oracle, with and without the pair cache:

* from rest, as configured: the first 12 steps (the initial detection bit
  for bit, then the pair lists and forces of every step);
* settled: the library's own steps pour the particles onto the floor wall
  (a contact-rich state with wall and particle contacts), then a fresh GPU
  simulation and the oracle start from that state for 12 steps.

Tolerances as in the other parity tests: contact lists equal (overlaps bit
for bit at the first detection, to 1e-9 relative afterwards), forces and
torques to 1e-10 relative to the largest entry, positions to 1e-13.
"""
import numpy as np
import pytest

from conftest import canonical, keys, rel_err
import parity_cases as PC

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def settled_pour(fundem):
    from fundem_b200 import workloads
    sc = PC.pour_config0()
    sim = fundem.Simulation.from_scenario(sc, records=False)
    sim.detect()
    rec = workloads.settle(sim, np.ones(len(sc.particles)), 5e-6, 30000)
    st = sim.state()
    sim.close()
    sc.particles.pos, sc.particles.vel, sc.particles.quat = st["pos"], st["vel"], st["quat"]
    return sc, rec


def _compare(fundem, oracle_mod, sc, cache, steps=12, min_contacts=0):
    g = fundem.Simulation.from_scenario(sc)
    g.set_pair_cache(1 if cache else 0)
    o = oracle_mod.OracleWorld.from_scenario(sc)
    g.detect()
    o.initial_detect()
    for k in range(2):
        a, b = canonical(g.contacts(k)), canonical(o.contacts(k))
        assert np.array_equal(keys(a), keys(b)), k
        assert np.array_equal(a["overlap"], b["overlap"]), k
    seen = 0
    for s in range(steps):
        g.step(1)
        o.step(1)
        for k in range(2):
            a, b = canonical(g.contacts(k)), canonical(o.contacts(k))
            assert np.array_equal(keys(a), keys(b)), (s, k)
            if len(b["overlap"]):
                assert rel_err(a["overlap"], b["overlap"]) < 1e-9, (s, k)
            seen += len(b["overlap"])
        sg, so = g.state(), o.state()
        assert rel_err(sg["force"], so["force"]) < 1e-10, s
        assert rel_err(sg["torque"], so["torque"]) < 1e-10, s
        assert rel_err(sg["pos"], so["pos"]) < 1e-13, s
        assert rel_err(sg["vel"], so["vel"]) < 1e-10, s
    g.sync()
    g.close()
    assert seen >= min_contacts
    return seen


@pytest.mark.parametrize("cache", [False, True])
def test_config0_from_rest_vs_oracle(fundem, oracle_mod, cache):
    sc = PC.pour_config0()
    assert len(sc.particles) == 1000 and len(sc.walls) == 6
    _compare(fundem, oracle_mod, sc, cache)


@pytest.mark.parametrize("cache", [False, True])
def test_config0_settled_vs_oracle(fundem, oracle_mod, settled_pour, cache):
    sc, rec = settled_pour
    # several hundred node contacts per step, walls included
    _compare(fundem, oracle_mod, sc, cache, min_contacts=12 * 300)
