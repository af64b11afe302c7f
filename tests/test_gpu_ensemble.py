"""Long runs against the CPU oracle: a 216-body cluster, compressed into
overlap inside an open box, expands, collides and settles under gravity.

DEM is chaotic, so the comparison has two parts: pointwise over the first
1,000 steps (states and contact sets), and beyond that through ensemble
statistics of the packing that do not depend on any one trajectory: the
mean coordination number, the height of the pile, the kinetic energy and
the distribution of contact overlaps (the normal-force distribution, since
the normal force is kn times the overlap plus damping)."""
import numpy as np
import pytest

from conftest import canonical, keys, rel_err
import parity_cases as PC

pytestmark = pytest.mark.gpu

N = 216


def _node_owner(sc):
    counts = [len(sc.particle_geometries[g].nodes) for g in sc.particles.geo]
    return np.repeat(np.arange(len(counts)), counts)


def _stats(state, contacts, owner, masses):
    """Coordination number (distinct touching partners per body, walls
    excluded), mean height, kinetic energy and the contact overlaps."""
    pairs = {(int(owner[m]), int(s)) for m, s in zip(contacts["master"], contacts["slave"])}
    coord = 2.0 * len(pairs) / len(state["pos"])
    ke = 0.5 * float(np.sum(masses * np.sum(state["vel"] ** 2, axis=1)))
    return coord, float(state["pos"][:, 2].mean()), ke, np.asarray(contacts["overlap"])


def _ks(a, b):
    """Two-sample Kolmogorov-Smirnov distance."""
    a, b = np.sort(a), np.sort(b)
    x = np.concatenate([a, b])
    fa = np.searchsorted(a, x, side="right") / len(a)
    fb = np.searchsorted(b, x, side="right") / len(b)
    return float(np.abs(fa - fb).max())


def test_long_run_pointwise_then_ensemble(fundem, oracle_mod):
    sc = PC.cluster(n=N)
    g = fundem.Simulation.from_scenario(sc)
    o = oracle_mod.OracleWorld.from_scenario(sc)
    g.detect()
    o.initial_detect()
    owner = _node_owner(sc)
    inv_mass = {int(k): g.geometry(int(k))["inv_mass"] for k in set(sc.particles.geo)}
    masses = np.array([1.0 / inv_mass[int(k)] for k in sc.particles.geo])
    done = 0
    # pointwise over the first 1,000 steps
    for s in (100, 250, 500, 1000):
        g.step(s - done)
        o.step(s - done)
        done = s
        sg, so = g.state(), o.state()
        assert rel_err(sg["pos"], so["pos"]) < 1e-11, s
        assert rel_err(sg["vel"], so["vel"]) < 1e-7, s
        for k in (0, 1):
            assert np.array_equal(keys(canonical(g.contacts(k))), keys(canonical(o.contacts(k)))), (s, k)
    # beyond: statistics of the packing
    for s in (2000, 3000, 4000):
        g.step(s - done)
        o.step(s - done)
        done = s
        cg, zg, kg, ovg = _stats(g.state(), g.contacts(0), owner, masses)
        co, zo, ko, ovo = _stats(o.state(), o.contacts(0), owner, masses)
        assert abs(cg - co) <= 0.05 * max(co, 1.0), (s, cg, co)
        assert abs(zg - zo) <= 1e-3 * abs(zo), (s, zg, zo)
        assert abs(kg - ko) <= 0.05 * max(ko, 1e-12), (s, kg, ko)
        if len(ovo) >= 20 and len(ovg) >= 20:
            assert _ks(ovg, ovo) < 0.1, s
        print(f"step {s}: coordination {cg:.3f} / {co:.3f}, mean z {zg:.6f} / {zo:.6f}, "
              f"kinetic energy {kg:.3e} / {ko:.3e}, contacts {len(ovg)} / {len(ovo)}")
    g.sync()
