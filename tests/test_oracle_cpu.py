"""CPU tests of the oracle: reference quirks, host setup arithmetic, analytic
known answers, and the pin against the reference's own build (golden
fixtures dumped from the reference CUDA build on a B200)."""
import hashlib

import numpy as np
import pytest

from conftest import canonical, golden_contacts, golden_state, keys, load_golden, rel_err, scenario_sha
import parity_cases as PC
from fundem_b200 import scenario as S


def test_inverse_det_threshold(oracle_mod):
    # myMat.h:175-179: |det| < 1e-30 -> zero matrix
    m = 1e-5
    I = 0.4 * m * (1e-3) ** 2
    assert np.all(oracle_mod.inverse_sym([I, I, I, 0, 0, 0]) == 0.0)
    inv = oracle_mod.inverse_sym([2.0, 3.0, 4.0, 0.1, 0.2, 0.3])
    A = np.array([[2.0, 0.1, 0.2], [0.1, 3.0, 0.3], [0.2, 0.3, 4.0]])
    B = np.array([[inv[0], inv[3], inv[4]], [inv[3], inv[1], inv[5]], [inv[4], inv[5], inv[2]]])
    assert np.allclose(A @ B, np.eye(3), atol=1e-14)


def test_mass_properties_sphere(oracle_mod):
    # smoothed-Heaviside mass of a sphere SDF approaches the analytic mass
    g = S.sphere_template(0.01, n=41, level=1)
    g.spacing = 0.01 / 10.0
    ax = (np.arange(41) - 20.0) * g.spacing
    Z, Y, X = np.meshgrid(ax, ax, ax, indexing="ij")
    sdf = (np.sqrt(X * X + Y * Y + Z * Z) - 0.01).reshape(-1)
    m, c, I = oracle_mod.mass_properties(1000.0, [ax[0]] * 3, g.spacing, [41, 41, 41], sdf)
    ma = 4.0 / 3.0 * np.pi * 0.01 ** 3 * 1000.0
    assert abs(m - ma) / ma < 2e-2
    assert np.abs(c).max() < 1e-12
    assert abs(I[0] - 0.4 * ma * 1e-4) / (0.4 * ma * 1e-4) < 4e-2
    # the vectorised restatement used by the scenario builder agrees
    m2, c2, I2 = S.mass_properties(1000.0, [ax[0]] * 3, g.spacing, [41, 41, 41], sdf)
    assert abs(m2 - m) / m < 1e-12 and np.allclose(I2, I, rtol=1e-10)


def test_sphere_bounce_energy_and_contact_time(oracle_mod):
    """apps/test/LSSphereBouncing.cpp: e = 1, kn = m pi^2 / (2 t_c^2).  Walls
    use the particle's kn unchanged (contactKernel.cu:196).  The app's node
    set puts six nodes on the south pole (theta = pi for every phi), so six
    node contacts act in parallel: the contact lasts pi sqrt(m / (6 kn)) and
    the rebound speed equals the impact speed."""
    sc = S.sphere_on_plane(height=0.02, dt_frac=200.0)
    w = oracle_mod.OracleWorld.from_scenario(sc)
    w.initial_detect()
    dt = sc.dt
    v_in = None
    t_in = t_out = None
    for k in range(3000):
        w.step(1)
        n = len(w.contacts(1)["master"])
        vz = w.state()["vel"][0, 2]
        if n and t_in is None:
            t_in, v_in = k * dt, vz
        if t_in is not None and n == 0 and t_out is None:
            t_out, v_out = k * dt, vz
            break
    assert t_in is not None and t_out is not None
    m = sc.particle_geometries[0].mass
    kn = sc.particle_materials[0][0]
    t_c = np.pi * np.sqrt(m / (6.0 * kn))
    assert abs((t_out - t_in) - t_c) < 2 * dt
    assert abs(abs(v_out) - abs(v_in)) / abs(v_in) < 0.02


def test_restitution_ratio(oracle_mod):
    """With e < 1 each node contact carries the damping c_n = 2 zeta sqrt(m kn),
    zeta = -ln e / sqrt(ln^2 e + pi^2) (contactKernel.cuh:50-53).  Six
    coincident pole nodes act in parallel, so the effective damping ratio is
    sqrt(6) zeta and the rebound/impact ratio is exp(-pi z / sqrt(1 - z^2))
    with z = sqrt(6) zeta (gravity off)."""
    sc = S.sphere_on_plane(height=0.0105, dt_frac=400.0)
    e = 0.5
    m0 = sc.particle_materials[0]
    sc.particle_materials = [(m0[0], m0[1], m0[2], e)]
    sc.wall_materials = [(0.0, 1.0)]
    sc.gravity = np.zeros(3)
    sc.particles.vel[0] = [0.0, 0.0, -0.5]
    w = oracle_mod.OracleWorld.from_scenario(sc)
    w.initial_detect()
    v_in = v_out = None
    for k in range(6000):
        w.step(1)
        n = len(w.contacts(1)["master"])
        vz = w.state()["vel"][0, 2]
        if n and v_in is None:
            v_in = vz
        if v_in is not None and n == 0:
            v_out = vz
            break
    assert v_out is not None
    lr = np.log(e)
    zeta = -lr / np.sqrt(lr * lr + np.pi ** 2)
    z = np.sqrt(6.0) * zeta
    expect = np.exp(-np.pi * z / np.sqrt(1 - z * z))
    assert abs(abs(v_out / -0.5) - expect) / expect < 0.03


def test_sliding_spring_coulomb_cap(oracle_mod):
    """A block pushed along a wall slides once the tangential spring force
    reaches mu |F_n| (integrateSlidingSpring, contactKernel.cuh:4-34): the
    decelerating force is mu * m * g."""
    sc = S.sphere_on_plane(height=0.1, dt_frac=200.0)
    mu = 0.3
    kn, ks = sc.particle_materials[0][0], 0.8 * sc.particle_materials[0][0]
    sc.particle_materials = [(kn, ks, mu, 0.2)]
    sc.wall_materials = [(mu, 0.2)]
    # rest the sphere on the plane with its lowest nodes just inside
    sc.particles.pos[0] = [0.0, 0.0, 0.0099]
    sc.particles.vel[0] = [0.5, 0.0, 0.0]
    sc.gravity = np.array([0.0, 0.0, -9.81])
    w = oracle_mod.OracleWorld.from_scenario(sc)
    w.initial_detect()
    dt = sc.dt
    w.step(200)
    v0 = w.state()["vel"][0, 0]
    w.step(200)
    v1 = w.state()["vel"][0, 0]
    decel = (v0 - v1) / (200 * dt)
    # inverse inertia is non-zero at this scale, so rolling takes over
    # part of the motion; the decelerating friction stays <= mu g
    assert 0.0 < decel <= mu * 9.81 * 1.05


def test_bond_elastic_response(oracle_mod):
    """Two bonded bodies pulled apart: the bond's normal force is B1 (D - D0)
    with B1 = E A / L (VBondedInteraction.h:133-148)."""
    sc = S.sphere_on_plane()
    g = sc.particle_geometries[0]
    sc.walls = S.Objects.empty()
    sc.wall_geometries = []
    sc.wall_materials = []
    sc.gravity = np.zeros(3)
    P = S.Objects(np.array([[0.0, 0.0, 0.0], [0.03, 0.0, 0.0]]), np.zeros((2, 3)), np.zeros((2, 3)),
                  np.array([[1.0, 0, 0, 0], [1.0, 0, 0, 0]]), np.zeros(2, np.int32), np.zeros(2, np.int32))
    sc.particles = P
    R, L0, E = 0.002, 0.01, 1e7
    sc.bonds = S.Bonds(np.array([0], np.int32), np.array([1], np.int32), np.array([[0.015, 0, 0]]),
                       np.array([[-1.0, 0, 0]]), np.array([R]), np.array([L0]), np.array([E]), np.array([0.3]),
                       np.zeros(1), np.zeros(1), np.zeros(1))
    sc.domain_min, sc.domain_max = np.array([-0.1, -0.1, -0.1]), np.array([0.1, 0.1, 0.1])
    w = oracle_mod.OracleWorld.from_scenario(sc)
    st = w.state()
    d = 1e-5
    st["pos"][1, 0] += d
    w.set_state(pos=st["pos"])
    w.detect_and_force()
    f = w.state()["force"]
    B1 = E * np.pi * R * R / L0
    assert abs(f[0, 0] - B1 * d) / (B1 * d) < 1e-6
    assert abs(f[1, 0] + B1 * d) / (B1 * d) < 1e-6


# ---------------------------------------------------------------------------
# pin against the reference's own CUDA build
# ---------------------------------------------------------------------------
# contact kinds as dumped (the sector images' lists only in sector runs)
KINDS = ("pp", "pw", "gx", "gy", "gxy", "gr90", "gr180", "gr270")


def _rebuild_and_check(name):
    g = load_golden(name)
    sha = scenario_sha(name)
    assert str(g["scenario_sha256"]) == sha, "scenario builder changed since the fixture was made"
    return g


@pytest.mark.parametrize("name", ["cluster", "periodic", "pour_mm", "sector", "pour1000"])
def test_oracle_geometry_matches_reference(oracle_mod, name):
    g = _rebuild_and_check(name)
    w = oracle_mod.OracleWorld.from_scenario(PC.CASES[name]())
    for k in range(len(g["geo_radius"])):
        og = w.geometry(k)
        assert og["radius"] == g["geo_radius"][k]
        assert og["inv_mass"] == pytest.approx(g["geo_inv_mass"][k], rel=1e-13)
        assert np.allclose(og["inertia"], g["geo_inertia"][k], rtol=1e-12, atol=0)
        assert np.allclose(og["inv_inertia"], g["geo_inv_inertia"][k], rtol=1e-10, atol=0)
    st = w.state()
    # the reference records positions after its pre-loop detection, whose
    # sector wrap has already turned bodies that start outside the sector
    sc = PC.CASES[name]()
    inside = ~((st["pos"][:, 0] < sc.domain_min[0]) | (st["pos"][:, 1] < sc.domain_min[1])) \
        if getattr(sc, "periodic_sector", False) else np.ones(len(st["pos"]), bool)
    assert rel_err(st["pos"][inside], g["geo_pos"][inside]) < 1e-15
    gr = w.grid()
    assert np.all(gr["size"] == g["geo_grid_size"])
    assert np.all(gr["inv_cell"] == g["geo_grid_inv"])


def _oracle_at(oracle_mod, name, g, step):
    """Oracle world holding the reference's state at the hook of `step`
    (positions, velocities after the first half kick, forces, history)."""
    w = oracle_mod.OracleWorld.from_scenario(PC.CASES[name]())
    st = golden_state(g, step)
    w.set_state(**st)
    w.set_state(wall=True, pos=g[f"s{step}_wall_pos"], quat=g[f"s{step}_wall_quat"])
    for kind_i, kind in enumerate(KINDS):
        if f"s{step}_{kind}_master" not in g:
            continue
        c = golden_contacts(g, step, kind)
        if len(c["master"]):
            w.set_contacts(kind_i, c["master"], c["slave"], c["spring"])
    act = g[f"s{step}_bond_activated"]
    if len(act):
        w.set_bond_activation(act)
    return w


@pytest.mark.parametrize("name", ["cluster", "periodic", "pour_mm", "sector", "pour1000"])
def test_oracle_detection_bit_exact_vs_reference(oracle_mod, name):
    """From the reference's exact state at step s, the oracle's detection
    reproduces the reference's contact set and overlaps bit for bit (the
    nvcc contraction pattern of the membership arithmetic is matched)."""
    g = _rebuild_and_check(name)
    steps = [int(s) for s in g["steps"]]
    checked = 0
    for s in steps:
        if s - 1 not in steps:
            continue
        w = _oracle_at(oracle_mod, name, g, s - 1)
        # replay step s: second half kick of s-1, then kick, drift, detection
        w.half_kick()
        w.front()
        w.detect_and_force()
        for kind_i, kind in enumerate(KINDS):
            if f"s{s}_{kind}_master" not in g:
                continue
            ref = canonical(golden_contacts(g, s, kind))
            got = canonical(w.contacts(kind_i))
            assert np.array_equal(keys(got), keys(ref)), (name, s, kind)
            if len(ref["overlap"]):
                assert rel_err(got["overlap"], ref["overlap"]) < 1e-9
                assert rel_err(got["spring"], ref["spring"]) < 1e-8
        st = w.state()
        ref = golden_state(g, s)
        assert rel_err(st["pos"], ref["pos"]) < 1e-12
        assert rel_err(st["force"], ref["force"]) < 1e-8
        assert rel_err(st["torque"], ref["torque"]) < 1e-8
        checked += 1
    assert checked > 0


@pytest.mark.parametrize("name", ["cluster", "pour_mm", "pour1000"])
def test_oracle_overlaps_bitwise_from_reference_state(oracle_mod, name):
    """Detection from the reference's dumped positions at step s (no
    integration in between): overlaps agree bit for bit."""
    g = _rebuild_and_check(name)
    s = int(g["steps"][1])
    w = _oracle_at(oracle_mod, name, g, s - 1)
    w.set_state(**golden_state(g, s))
    w.detect_and_force()
    ref = canonical(golden_contacts(g, s, "pp"))
    got = canonical(w.contacts(0))
    assert np.array_equal(keys(got), keys(ref))
    if len(ref["overlap"]):
        assert np.array_equal(got["overlap"], ref["overlap"])
        assert np.abs(got["normal"] - ref["normal"]).max() < 1e-14


def test_oracle_sector_trajectory_vs_reference(oracle_mod):
    """Sector periodicity over the whole fixture horizon from t = 0: every
    contact list, the turned images' included, and the positions follow the
    reference build (the body that starts outside the x face is turned back
    in on the first step)."""
    g = _rebuild_and_check("sector")
    w = oracle_mod.OracleWorld.from_scenario(PC.CASES["sector"]())
    w.initial_detect()
    done = 0
    for s in [int(x) for x in g["steps"]]:
        w.step(s - done)
        done = s
        assert rel_err(w.state()["pos"], golden_state(g, s)["pos"]) < 1e-14, s
        for kind_i, kind in enumerate(KINDS):
            if kind in ("gx", "gy", "gxy"):
                continue
            got = keys(canonical(w.contacts(kind_i)))
            assert np.array_equal(got, keys(canonical(golden_contacts(g, s, kind)))), (s, kind)
            if kind_i >= 5:
                assert len(got) > 0, (s, kind)
