"""Edge cases of the timestep on the GPU, against the oracle where there is
a result to compare: no particles, no walls, partners outside the domain
(invisible, mySpatialGrid.cu:17-22), a particle with more partners than a
segment holds (reported, not silent), an empty step, and a state round
trip."""
import numpy as np
import pytest

from fundem_b200 import scenario as S
from conftest import canonical

pytestmark = pytest.mark.gpu


def _spheres(pos, radius=0.01, walls=True, domain=((-0.1, -0.1, -0.1), (0.1, 0.1, 0.1))):
    n = len(pos)
    m = 4.0 / 3.0 * np.pi * radius ** 3 * 2000.0
    I = 0.4 * m * radius * radius
    geo = S.sphere_template(radius, mass=m, inertia=[I, I, I, 0, 0, 0])
    objs = S.Objects(np.asarray(pos, float), np.zeros((n, 3)), np.zeros((n, 3)),
                     np.tile([1.0, 0, 0, 0], (n, 1)), np.zeros(n, np.int32), np.zeros(n, np.int32))
    if walls:
        wg = [S.plane_wall_template(0.4)]
        wo = S.Objects(np.array([[0.0, 0.0, -0.05]]), np.zeros((1, 3)), np.zeros((1, 3)),
                       np.array([S.WALL_QUAT["+z"]]), np.zeros(1, np.int32), np.zeros(1, np.int32))
    else:
        wg, wo = [], S.Objects.empty()
    return S.Scenario(domain_min=np.array(domain[0]), domain_max=np.array(domain[1]),
                      gravity=np.array([0.0, 0.0, -9.81]), dt=1e-5,
                      particle_materials=[(1e4, 0.8e4, 0.5, 0.5)], wall_materials=[(0.5, 0.5)],
                      particle_geometries=[geo], wall_geometries=wg, particles=objs, walls=wo, name="edges")


def _same_contacts(g, o, kinds=(0, 1)):
    for k in kinds:
        a, b = canonical(g.contacts(k)), canonical(o.contacts(k))
        assert np.array_equal(a["master"], b["master"]) and np.array_equal(a["slave"], b["slave"])
        assert np.array_equal(a["overlap"], b["overlap"])


def test_walls_only(fundem):
    sc = _spheres(np.zeros((0, 3)))
    s = fundem.Simulation.from_scenario(sc)
    s.detect()
    s.step(5)
    s.sync()
    assert s.num(False) == 0 and s.num_contacts(fundem.PP) == 0 and s.num_contacts(fundem.PW) == 0
    s.close()


def test_no_walls_against_oracle(fundem, oracle_mod):
    sc = _spheres([[0.0, 0.0, 0.0], [0.0195, 0.0, 0.0], [0.0, 0.0196, 0.0]], walls=False)
    g = fundem.Simulation.from_scenario(sc)
    o = oracle_mod.OracleWorld.from_scenario(sc)
    g.detect(); o.initial_detect()
    _same_contacts(g, o, kinds=(0,))
    assert g.num_contacts(fundem.PP) > 0
    g.step(3); o.step(3)
    a, b = g.state(), o.state()
    assert np.abs(a["pos"] - b["pos"]).max() < 1e-13
    g.close()


def test_partner_outside_domain_is_invisible(fundem, oracle_mod):
    # particle 1 overlaps particle 0 but its centre lies outside the domain:
    # it gets no cell and is nobody's partner; particle 0's centre is inside
    sc = _spheres([[0.0, 0.0, 0.095], [0.0, 0.0, 0.114]], walls=False,
                  domain=((-0.1, -0.1, -0.1), (0.1, 0.1, 0.1)))
    g = fundem.Simulation.from_scenario(sc)
    o = oracle_mod.OracleWorld.from_scenario(sc)
    g.detect(); o.initial_detect()
    assert g.num_contacts(fundem.PP) == 0
    _same_contacts(g, o, kinds=(0,))
    g.close()


def test_too_many_partners_is_reported(fundem):
    # a large sphere (index 0) with 100 small ones of higher index on a shell
    # just inside touching distance: more partners than a segment holds (64),
    # which the step reports instead of dropping them silently
    R, r = 0.05, 0.005
    golden = np.pi * (3.0 - np.sqrt(5.0))
    k = np.arange(100)
    z = 1.0 - 2.0 * (k + 0.5) / 100
    ring = np.stack([np.sqrt(1 - z * z) * np.cos(golden * k), np.sqrt(1 - z * z) * np.sin(golden * k), z], 1)
    ring *= R + 0.98 * r
    sc = _spheres(np.vstack([[0.0, 0.0, 0.0], ring]), walls=False, domain=((-0.2, -0.2, -0.2), (0.2, 0.2, 0.2)))
    mb = 4.0 / 3.0 * np.pi * R ** 3 * 2000.0
    big = S.sphere_template(R, mass=mb, inertia=[0.4 * mb * R * R] * 3 + [0, 0, 0])
    ms = 4.0 / 3.0 * np.pi * r ** 3 * 2000.0
    small = S.sphere_template(r, mass=ms, inertia=[0.4 * ms * r * r] * 3 + [0, 0, 0])
    sc.particle_geometries = [big, small]
    sc.particles.geo = np.array([0] + [1] * 100, np.int32)
    s = fundem.Simulation.from_scenario(sc)
    with pytest.raises(fundem.FundemError):
        s.detect()
        s.step(1)
        s.sync()
    s.close()


def test_zero_steps_and_state_round_trip(fundem):
    sc = _spheres([[0.0, 0.0, 0.0], [0.03, 0.0, 0.0]])
    s = fundem.Simulation.from_scenario(sc)
    s.detect()
    st = s.state()
    s.step(0)
    s.sync()
    st2 = s.state()
    for k in st:
        assert np.array_equal(st[k], st2[k])
    s.set_state(pos=st["pos"] + 1e-3, vel=st["vel"] + 0.5)
    st3 = s.state()
    assert np.array_equal(st3["pos"], st["pos"] + 1e-3) and np.array_equal(st3["vel"], st["vel"] + 0.5)
    s.close()
