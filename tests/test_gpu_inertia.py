"""The physical inverse-inertia rule on the GPU against the CPU oracle: the
mm-scale pour, whose bodies never turn under the reference's inverse()
(|det I| < 1e-30 gives zero, myMat.h:163-194), turns under contact torques
here, and every list, force, torque and state follows the oracle at the
tolerances of the other parity tests."""
import dataclasses

import numpy as np
import pytest

from conftest import canonical, keys, rel_err
import parity_cases as PC

pytestmark = pytest.mark.gpu


def _pair(fundem, oracle_mod, inertia="physical"):
    sc = dataclasses.replace(PC.pour_mm(), inertia=inertia)
    return sc, fundem.Simulation.from_scenario(sc), oracle_mod.OracleWorld.from_scenario(sc)


def test_physical_inverse_matches_oracle(fundem, oracle_mod):
    sc, g, o = _pair(fundem, oracle_mod)
    for k in range(len(sc.particle_geometries)):
        got, ref = g.geometry(k)["inv_inertia"], o.geometry(k)["inv_inertia"]
        assert np.any(ref)
        assert np.array_equal(got, ref)
    g.close()


def test_physical_steps_vs_oracle(fundem, oracle_mod):
    sc, g, o = _pair(fundem, oracle_mod)
    g.detect()
    o.initial_detect()
    w0 = g.state()["angvel"].copy()
    for s in range(20):
        g.step(1)
        o.step(1)
        for k in range(2):
            a, b = canonical(g.contacts(k)), canonical(o.contacts(k))
            assert np.array_equal(keys(a), keys(b)), (s, k)
            if len(b["overlap"]):
                assert rel_err(a["overlap"], b["overlap"]) < 1e-9
        sg, so = g.state(), o.state()
        assert rel_err(sg["force"], so["force"]) < 1e-10
        assert rel_err(sg["torque"], so["torque"]) < 1e-10
        assert rel_err(sg["pos"], so["pos"]) < 1e-13
        assert rel_err(sg["vel"], so["vel"]) < 1e-10
        assert rel_err(sg["angvel"], so["angvel"]) < 1e-10
        assert rel_err(sg["quat"], so["quat"]) < 1e-13
    # the bodies did turn
    assert np.abs(g.state()["angvel"] - w0).max() > 0.0
    g.sync()
    g.close()


def test_mode_takes_effect_at_the_next_setup(fundem, oracle_mod):
    """A simulation set up under the reference rule keeps every angular
    velocity; after a switch and a second setup (a new solve phase) its
    geometries carry the oracle's physical inverse and its bodies turn."""
    sc, g, _ = _pair(fundem, oracle_mod, inertia="reference")
    g.detect()
    w0 = g.state()["angvel"].copy()
    g.step(5)
    assert np.array_equal(g.state()["angvel"], w0)
    g.set_inertia_mode(fundem.INERTIA_PHYSICAL)
    g.setup(sc.domain_min, sc.domain_max)
    o = oracle_mod.OracleWorld.from_scenario(dataclasses.replace(sc, inertia="physical"))
    for k in range(len(sc.particle_geometries)):
        assert np.array_equal(g.geometry(k)["inv_inertia"], o.geometry(k)["inv_inertia"])
    g.detect()
    g.step(5)
    assert np.abs(g.state()["angvel"] - w0).max() > 0.0
    g.sync()
    g.close()
