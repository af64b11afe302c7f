"""GPU known-answer tests of the contact law, the integrator and bonds,
run through the C ABI (the same cases the oracle's CPU tests check)."""
import numpy as np
import pytest

from fundem_b200 import scenario as S

pytestmark = pytest.mark.gpu


def _bounce(fundem, e, gravity):
    sc = S.sphere_on_plane(height=0.0105, dt_frac=400.0)
    m0 = sc.particle_materials[0]
    sc.particle_materials = [(m0[0], m0[1], m0[2], e)]
    sc.wall_materials = [(0.0, 1.0)]
    sc.gravity = np.asarray(gravity, float)
    sc.particles.vel[0] = [0.0, 0.0, -0.5]
    g = fundem.Simulation.from_scenario(sc)
    g.detect()
    t_in = t_out = v_in = v_out = None
    for k in range(4000):
        g.step(1)
        n = g.num_contacts(1)
        vz = g.state()["vel"][0, 2]
        if n and t_in is None:
            t_in, v_in = k, vz
        if t_in is not None and n == 0:
            t_out, v_out = k, vz
            break
    g.sync()
    return sc, t_in, t_out, v_in, v_out


def test_elastic_bounce(fundem):
    """e = 1: six coincident pole nodes in parallel, contact time
    pi sqrt(m / (6 kn)), rebound speed equals the impact speed."""
    sc, t_in, t_out, v_in, v_out = _bounce(fundem, 1.0, [0, 0, 0])
    m = sc.particle_geometries[0].mass
    kn = sc.particle_materials[0][0]
    tc = np.pi * np.sqrt(m / (6 * kn))
    assert abs((t_out - t_in) * sc.dt - tc) < 2 * sc.dt
    assert abs(abs(v_out) - 0.5) / 0.5 < 0.01


def test_restitution(fundem):
    sc, t_in, t_out, v_in, v_out = _bounce(fundem, 0.5, [0, 0, 0])
    lr = np.log(0.5)
    z = np.sqrt(6.0) * (-lr / np.sqrt(lr * lr + np.pi ** 2))
    expect = np.exp(-np.pi * z / np.sqrt(1 - z * z))
    assert abs(abs(v_out / 0.5) - expect) / expect < 0.03


def test_bond_normal_stiffness(fundem):
    sc = S.sphere_on_plane()
    sc.walls = S.Objects.empty()
    sc.wall_geometries, sc.wall_materials = [], []
    sc.gravity = np.zeros(3)
    sc.particles = S.Objects(np.array([[0.0, 0.0, 0.0], [0.03, 0.0, 0.0]]), np.zeros((2, 3)), np.zeros((2, 3)),
                             np.array([[1.0, 0, 0, 0], [1.0, 0, 0, 0]]), np.zeros(2, np.int32), np.zeros(2, np.int32))
    R, L0, E = 0.002, 0.01, 1e7
    sc.bonds = S.Bonds(np.array([0], np.int32), np.array([1], np.int32), np.array([[0.015, 0, 0]]),
                       np.array([[-1.0, 0, 0]]), np.array([R]), np.array([L0]), np.array([E]), np.array([0.3]),
                       np.zeros(1), np.zeros(1), np.zeros(1))
    sc.domain_min, sc.domain_max = np.array([-0.1, -0.1, -0.1]), np.array([0.1, 0.1, 0.1])
    g = fundem.Simulation.from_scenario(sc)
    st = g.state()
    d = 1e-5
    st["pos"][1, 0] += d
    g.set_state(pos=st["pos"])
    g.step_begin(dt=1e-9)
    f = g.state()["force"]
    B1 = E * np.pi * R * R / L0
    assert abs(f[0, 0] - B1 * d) / (B1 * d) < 1e-3
    assert abs(f[1, 0] + B1 * d) / (B1 * d) < 1e-3
    g.sync()


def test_free_flight_integration(fundem):
    """Without contacts the half-kick / drift scheme integrates gravity
    exactly: z(t) = z0 + v0 t - g t^2 / 2 at the step boundaries."""
    sc = S.sphere_on_plane(height=0.5)
    sc.particles.vel[0] = [0.1, 0.0, 2.0]
    g = fundem.Simulation.from_scenario(sc)
    g.detect()
    n = 500
    g.step(n)
    st = g.state()
    t = n * sc.dt
    assert abs(st["pos"][0, 2] - (0.5 + 2.0 * t - 0.5 * 9.81 * t * t)) < 1e-12
    assert abs(st["pos"][0, 0] - 0.1 * t) < 1e-12
    g.sync()
