"""Independent simulations tiled into one (fundem_b200.batch.TiledBatch): one
launch per stage serves every simulation, each with its own material block
and its own walls (per-particle wall groups).  Each simulation of the tiled
run must evolve as it does alone: the same contact sets and positions to
1e-12 relative after 120 steps (the cell grids of the two runs differ, so
sums are not compared bit for bit), and the parameter gradients of the tiled
run's adjoint are each simulation's own."""
import numpy as np
import pytest

from conftest import canonical, keys, rel_err

pytestmark = pytest.mark.gpu


def test_tiled_batch_equals_solo_runs(fundem):
    from fundem_b200 import batch
    scs, params = batch.calibration_scenarios(n_sims=6, seed=4, n_min=300, n_max=1500)
    rng = np.random.default_rng(4)
    for sc in scs:
        # lattices pulled 4% towards the centre of their floor, small random
        # velocities: contacts from the first steps, with one another and
        # with the floor wall
        P = sc.particles
        c = 0.5 * (P.pos.min(axis=0) + P.pos.max(axis=0))
        c[2] = 0.0
        P.pos[:] = c + (P.pos - c) * 0.96
        P.vel[:] = rng.normal(0.0, 0.05, P.vel.shape)
    tb = batch.TiledBatch(scs)
    tb.run(120)
    tiled = tb.states()
    pp = tb.sim.contacts(fundem.PP)
    pw = tb.sim.contacts(fundem.PW)
    layout, tsc = tb.layout, tb.scenario
    tb.close()
    total_pp = total_pw = 0
    for i, sc in enumerate(scs):
        s = fundem.Simulation.from_scenario(sc, records=False)
        s.detect()
        s.step(120)
        st = s.state()
        assert rel_err(tiled[i]["pos"], st["pos"]) < 1e-12, i
        assert rel_err(tiled[i]["vel"], st["vel"]) < 1e-9, i
        total_pp += s.num_contacts(fundem.PP)
        total_pw += s.num_contacts(fundem.PW)
        s.close()
    assert len(pp["master"]) == total_pp and len(pw["master"]) == total_pw and total_pw > 0
    # every contact joins a particle to a particle or wall of its own simulation
    counts = np.array([len(tsc.particle_geometries[g].nodes) for g in tsc.particles.geo], np.int64)
    node_base = np.concatenate([[0], np.cumsum(counts)[:-1]])
    p_start = np.array([p0 for (p0, _) in layout["particles"]])
    w_start = np.array([w0 for (w0, _) in layout["walls"]])
    sim_of_particle = lambda idx: np.searchsorted(p_start, idx, side="right") - 1
    owner = np.searchsorted(node_base, pp["master"], side="right") - 1
    assert np.array_equal(sim_of_particle(owner), sim_of_particle(pp["slave"]))
    owner_w = np.searchsorted(node_base, pw["master"], side="right") - 1
    assert np.array_equal(sim_of_particle(owner_w), np.searchsorted(w_start, pw["slave"], side="right") - 1)
