"""The pair cache of the particle-particle list (fundem_set_pair_cache) on the
GPU.  Cached steps keep the candidate pairs and contact slots of the last
rebuild and run the exact double-precision node predicate on every slot, so
the contact lists must be the ones a full detection gives:

* against the CPU oracle, step by step on the fixture cases (walls, periodic
  ghosts, millimetre pour, and a tall periodic column whose upper images the
  reference hashes into clamped cells), with the tolerances of the uncached
  parity tests:
  contact lists equal, overlaps to 1e-9 relative, forces and torques to 1e-10
  relative to the largest entry, positions to 1e-13;
* against the same run without the cache on a settled, bonded slab of the
  benchmark column: identical contact lists at every check over 300 steps,
  forces to 1e-9 (only the order of the per-pair force sums differs, since
  the cached slot layout holds extra candidate nodes);
* graph replays with the cache equal plain cached stepping bit for bit.
"""
import numpy as np
import pytest

from conftest import canonical, keys, rel_err
import parity_cases as PC

pytestmark = pytest.mark.gpu

CASES = ["cluster", "periodic", "pour_mm", "periodic_tall", "periodic_tall_nocache"]


def _case(name):
    if name.startswith("periodic_tall"):
        # a periodic column taller than it is wide: images of the upper
        # bodies lie above max y, which the reference's ghost hash tests z
        # against (they go to a clamped cell), so those steps build the
        # ghost lists without the cache
        return PC.periodic(nx=2, ny=2, nz=6)
    return PC.CASES[name]()


def _same_lists(got, ref, what=""):
    got, ref = canonical(got), canonical(ref)
    kg, kr = keys(got), keys(ref)
    if not np.array_equal(kg, kr):
        sg, sr = set(map(tuple, kg.tolist())), set(map(tuple, kr.tolist()))
        raise AssertionError(f"{what}: {len(kg)} contacts against {len(kr)}; only here {sorted(sg - sr)[:8]}, "
                             f"only in the reference {sorted(sr - sg)[:8]}")
    if len(ref["overlap"]):
        assert rel_err(got["overlap"], ref["overlap"]) < 1e-9


@pytest.mark.parametrize("name", CASES)
def test_cached_steps_vs_oracle(fundem, oracle_mod, name):
    sc = _case(name)
    g = fundem.Simulation.from_scenario(sc)
    r = max(g.geometry(k)["radius"] for k in range(len(sc.particle_geometries)))
    cached = not name.endswith("nocache")   # the same case without the cache, for comparison
    g.set_pair_cache(1 if cached else 0, 0.05 * r)
    o = oracle_mod.OracleWorld.from_scenario(sc)
    g.detect()
    o.initial_detect()
    for s in range(30):
        g.step(1)
        o.step(1)
        for k in range(5):
            _same_lists(g.contacts(k), o.contacts(k), f"step {s}, kind {k}")
        sg, so = g.state(), o.state()
        assert rel_err(sg["force"], so["force"]) < 1e-10, s
        assert rel_err(sg["torque"], so["torque"]) < 1e-10, s
        assert rel_err(sg["pos"], so["pos"]) < 1e-13, s
    if len(sc.bonds):
        assert np.array_equal(g.bonds()["activated"], o.bonds()["activated"])
    rebuilds, steps, skin = g.pair_cache_stats()
    if cached:
        assert steps == 30 and skin == pytest.approx(0.05 * r) and 1 <= rebuilds <= 30
    g.sync()


def test_cached_equals_full_detection_on_settled_slab(fundem):
    from fundem_b200 import workloads
    sim, sc, info = workloads.bonded_column(n=2048, footprint=(16, 16), seed=3)
    sim.close()
    assert info["settled"]
    sims = {}
    for mode in (0, 1):
        s = fundem.Simulation.from_scenario(sc, records=False)
        s.set_pair_cache(mode)
        s.detect()
        sims[mode] = s
    sims[1].set_profiling(False, counters=True)
    sims[1].work_counters()
    n_checked = 0
    for block in range(15):
        for s in sims.values():
            s.step(20)
        a, b = sims[0].contacts(fundem.PP), sims[1].contacts(fundem.PP)
        assert len(a["master"]) > 500
        assert np.array_equal(keys(canonical(a)), keys(canonical(b))), block
        for k in (fundem.PW, fundem.GX, fundem.GY, fundem.GXY):
            assert np.array_equal(keys(canonical(sims[0].contacts(k))), keys(canonical(sims[1].contacts(k))))
        sa, sb = sims[0].state(), sims[1].state()
        assert rel_err(sb["force"], sa["force"]) < 1e-9, block
        assert rel_err(sb["pos"], sa["pos"]) < 1e-12, block
        assert np.array_equal(sims[0].bonds()["activated"], sims[1].bonds()["activated"])
        n_checked += 1
    wc = sims[1].work_counters()
    sims[1].set_profiling(False)
    # carried steps skip most slots by the slot bound and test the rest
    assert wc[5] > 0 and wc[6] > 0, wc
    print(f"cached predicate pass: {wc[5]} slots tested, {wc[6]} skipped by the slot bound")
    rebuilds, steps, _ = sims[1].pair_cache_stats()
    assert steps == 300
    # the platen moves the top of the slab by 0.5 um per step: the cache is
    # rebuilt every few steps there, and carried in between
    assert rebuilds < steps // 2, rebuilds
    for s in sims.values():
        s.sync()
        s.close()


def test_cached_graph_replay_equals_plain_steps(fundem):
    from fundem_b200 import workloads
    sim, sc, info = workloads.bonded_column(n=2048, footprint=(16, 16), seed=5)
    sim.close()
    out = []
    for use_graph in (False, True):
        s = fundem.Simulation.from_scenario(sc, records=False)
        s.set_pair_cache(1)
        s.detect()
        for _ in range(6):
            if use_graph:
                s.step_graph(25)
            else:
                s.step(25)
        s.sync()
        out.append((s.state(), s.contacts(fundem.PP)))
        s.close()
    (sa, ca), (sb, cb) = out
    for k in ("pos", "vel", "force"):
        assert np.array_equal(sa[k], sb[k]), k
    assert np.array_equal(keys(canonical(ca)), keys(canonical(cb)))
