"""A settled, bonded slab of the config-1 workload against the CPU oracle
until bonds break.

workloads.bonded_column builds the slab as it builds config 1 (superellipsoids
from 8 templates on a jittered lattice, periodic in x and y, settled under
gravity with the library's own steps, V-bonds across the small gaps, the top
platen started downward), here 2,048 particles on a 16 x 16 footprint.  The
platen runs at 20 m/s instead of 1 m/s so that bonds under it break within a
few hundred steps.  The GPU simulation and the oracle start from the
returned scenario (the same state, no contact history) and run in blocks of
10 steps; after every block the bond activation flags are equal bit for bit
(the reference breaks bonds in contactKernel.cu:333-342 and
contactKernel.cuh:190-198), the particle-particle contact lists are equal
and positions agree to 1e-12 relative.  The run stops 50 steps after the
first break."""
import numpy as np
import pytest

from conftest import canonical, keys, rel_err

pytestmark = pytest.mark.gpu


def test_bonded_slab_breaks_bonds_like_the_oracle(fundem, oracle_mod):
    from fundem_b200 import workloads
    sim, sc, info = workloads.bonded_column(n=2048, footprint=(16, 16), seed=3, platen_speed=20.0)
    sim.close()
    assert info["settled"]
    g = fundem.Simulation.from_scenario(sc, records=False)
    o = oracle_mod.OracleWorld.from_scenario(sc)
    g.detect()
    o.initial_detect()
    nb0 = int(np.sum(g.bonds()["activated"]))
    assert nb0 > 1000
    first_break = None
    for block in range(100):
        g.step(10)
        o.step(10)
        bg, bo = g.bonds()["activated"], o.bonds()["activated"]
        assert np.array_equal(bg, bo), (block, int(bg.sum()), int(bo.sum()))
        cg, co = canonical(g.contacts(fundem.PP)), canonical(o.contacts(fundem.PP))
        assert np.array_equal(keys(cg), keys(co)), block
        sg, so = g.state(), o.state()
        assert rel_err(sg["pos"], so["pos"]) < 1e-12, block
        if first_break is None and bg.sum() < nb0:
            first_break = block
        if first_break is not None and block >= first_break + 5:
            break
    g.sync()
    assert first_break is not None, "no bond broke within 1,000 steps"
    print(f"{nb0} bonds, first break in steps {10 * first_break + 1}-{10 * first_break + 10}, "
          f"{nb0 - int(bg.sum())} broken after {10 * (block + 1)} steps")
