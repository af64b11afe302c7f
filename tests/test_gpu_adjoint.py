"""The adjoint of the FP64 step (fundem_adjoint_*) against central finite
differences of the forward run, on bonded periodic columns (particle pairs,
floor and moving platen, periodic ghosts, bonds) of 512 translating
particles, over 50 steps in four checkpoint segments, for four seeds.

Loss: L = sum(w * x_T) + sum(u * v_T) with fixed random weights.  Gradients
with respect to the particle material's kn, ks, damping ratio and friction
coefficient (relative step 1e-4) and to initial velocity components
(step 1e-4 m/s) agree within 1e-3 relative.

The adjoint freezes the contact topology of each step.  A damped contact
starts with a finite force (the dashpot acts at zero overlap), so a
perturbation that moves a contact's first step changes the loss by a jump
that no derivative describes; over longer horizons the finite differences
cross such events (at 200 steps of this column they differ from the
frozen-topology gradient by several times).  Even at 50 steps a step of
1e-4 can reach one on one side: the forward and backward one-sided
differences then disagree, and the gradient is compared with the side that
stays smooth (its truncation error is of order h, 1e-4 relative).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

T, K = 50, 16


@pytest.fixture(scope="module", params=[11, 12, 13, 14])
def setup(fundem, request):
    from fundem_b200 import workloads
    sim, sc, info = workloads.bonded_column(n=512, footprint=(8, 8), seed=request.param)
    sim.close()
    # walls with more friction and restitution than the particles: the
    # particle-wall contacts then take mu = min(...) and e = min(...) from the
    # particle material, away from the kink where the two are equal
    sc.wall_materials = [(0.7, 0.9)]
    rng = np.random.default_rng(request.param)
    w = rng.standard_normal((512, 3))
    u = rng.standard_normal((512, 3)) * 1e-3
    return sc, w, u


def _with(sc, kn=None, ks=None, zeta=None, mu=None, dv=None):
    import copy
    s2 = copy.deepcopy(sc)
    kn0, ks0, mu0, e0 = s2.particle_materials[0]
    if zeta is not None:
        e0 = float(np.exp(-np.pi * zeta / np.sqrt(1.0 - zeta * zeta)))
    s2.particle_materials[0] = (kn if kn is not None else kn0, ks if ks is not None else ks0,
                                mu if mu is not None else mu0, e0)
    if dv is not None:
        s2.particles.vel = s2.particles.vel + dv
    return s2


def _loss(fundem, sc, w, u):
    s = fundem.Simulation.from_scenario(sc, records=False)
    s.detect()
    s.step(T)
    s.sync()
    st = s.state()
    s.close()
    return float(np.sum(w * st["pos"]) + np.sum(u * st["vel"])), st


def _check_fd(name, g, L0, Lp, Lm, h, atol):
    central = (Lp - Lm) / (2 * h)
    fwd, bwd = (Lp - L0) / h, (L0 - Lm) / h
    if abs(fwd - bwd) <= 1e-2 * abs(central) + atol:
        assert abs(g - central) <= 1e-3 * abs(central) + atol, (name, g, central)
    else:  # an event inside [x - h, x + h]: one side is smooth
        assert min(abs(g - fwd) - 1e-3 * abs(fwd), abs(g - bwd) - 1e-3 * abs(bwd)) <= atol, (name, g, fwd, bwd)


def _zeta(e):
    lr = np.log(e)
    return -lr / np.sqrt(lr * lr + np.pi * np.pi)


def test_adjoint_matches_finite_differences(fundem, setup):
    sc, w, u = setup
    L0, st_plain = _loss(fundem, sc, w, u)
    s = fundem.Simulation.from_scenario(sc, records=False)
    s.detect()
    s.adjoint_begin(K)
    s.adjoint_forward(T)
    st_adj = s.state()
    assert np.array_equal(st_adj["pos"], st_plain["pos"])  # recording does not change the run
    assert s.num_contacts(fundem.PP) + s.num_contacts(fundem.PW) > 0
    gv0, gp = s.adjoint_backward(w, u)
    st_after = s.state()
    assert np.array_equal(st_after["pos"], st_plain["pos"])  # final state restored
    s.adjoint_end()
    s.close()

    kn0, ks0, mu0, e0 = sc.particle_materials[0]
    checks = [("kn", dict(kn=kn0), kn0, gp[0, 0]), ("ks", dict(ks=ks0), ks0, gp[0, 1]),
              ("zeta", dict(zeta=_zeta(e0)), _zeta(e0), gp[0, 2]), ("mu", dict(mu=mu0), mu0, gp[0, 3])]
    for name, kw, x0, g in checks:
        h = 1e-4 * x0
        (k, _), = kw.items()
        Lp, _ = _loss(fundem, _with(sc, **{k: x0 + h}), w, u)
        Lm, _ = _loss(fundem, _with(sc, **{k: x0 - h}), w, u)
        _check_fd(name, g, L0, Lp, Lm, h, 1e-12)

    # initial velocities of the particles that moved most
    moved = np.argsort(-np.linalg.norm(st_plain["vel"], axis=1))[:2]
    for i in moved:
        for c in range(3):
            dv = np.zeros((512, 3))
            h = 1e-4
            dv[i, c] = h
            Lp, _ = _loss(fundem, _with(sc, dv=dv), w, u)
            Lm, _ = _loss(fundem, _with(sc, dv=-dv), w, u)
            _check_fd((i, c), gv0[i, c], L0, Lp, Lm, h, 1e-9)


def test_adjoint_refuses_rotating_bodies(fundem):
    import parity_cases
    sc = parity_cases.sphere()  # a 1 cm sphere: nonzero inverse inertia
    s = fundem.Simulation.from_scenario(sc)
    s.detect()
    with pytest.raises(fundem.FundemError):
        s.adjoint_begin(10)
    s.close()


def test_checkpoint_interval_autotuner(fundem):
    """The autotuner times forward + backward for several checkpoint
    intervals and picks one; the gradients do not depend on the interval,
    since each segment's re-run repeats the forward run (they agree to
    rounding: the reverse sweep adds to particles with atomics)."""
    from fundem_b200 import autotune, workloads
    sim, sc, info = workloads.bonded_column(n=512, footprint=(8, 8), seed=11)
    sim.close()
    rng = np.random.default_rng(5)
    w = rng.standard_normal((512, 3))
    u = rng.standard_normal((512, 3)) * 1e-3

    def make():
        s = fundem.Simulation.from_scenario(sc, records=False)
        s.detect()
        return s

    best, times = autotune.checkpoint_interval(make, 40, w, u, candidates=(5, 10, 20, 40))
    assert best in (5, 10, 20, 40) and set(times) == {5, 10, 20, 40}
    grads = []
    for k in (5, 40):
        s = make()
        s.adjoint_begin(k)
        s.adjoint_forward(40)
        grads.append(s.adjoint_backward(w, u))
        s.adjoint_end()
        s.close()
    for a, b in zip(grads[0], grads[1]):
        assert np.abs(a - b).max() <= 1e-10 * np.abs(b).max()


def _translating_periodic():
    """The periodic bonded parity case with zero inertia: cm bodies that
    translate and keep their initial angular velocities (about 10 rad/s)."""
    import copy
    import parity_cases
    sc = copy.deepcopy(parity_cases.periodic())
    for g in sc.particle_geometries:
        g.inertia = np.zeros(6)
    sc.wall_materials = [(0.7, 0.9)]
    return sc


def _turning_column():
    """The 512-particle bonded column with constant angular velocities: the
    particles spin at about 20 rad/s (zero inverse inertia keeps it) and the
    floor turns about z at 5 rad/s."""
    from fundem_b200 import workloads
    sim, sc, info = workloads.bonded_column(n=512, footprint=(8, 8), seed=12)
    sim.close()
    sc.wall_materials = [(0.7, 0.9)]
    rng = np.random.default_rng(12)
    sc.particles.angvel = rng.normal(0.0, 20.0, (len(sc.particles), 3))
    floor = int(np.argmin(sc.walls.pos[:, 2]))
    sc.walls.angvel = np.array(sc.walls.angvel, float, copy=True)
    sc.walls.angvel[floor] = [0.0, 0.0, 5.0]
    return sc


@pytest.mark.parametrize("case,steps", [("column", 50), ("column", 200), ("periodic", 60)])
def test_adjoint_matches_tangent_reference(fundem, oracle_mod, case, steps):
    """The reverse sweep against the FP64 CPU reference derivative
    (oracle/tangent.py: forward mode along the oracle's own run, with the
    same frozen topology).  Both are derivatives of the same model, so they
    agree to 1e-6 relative however many contact events the window holds,
    where finite differences stop describing it.  The cases carry turning
    bodies and a turning wall, so the contact velocity's dependence on the
    contact point enters, and the bonds' frame differences change each
    step."""
    from oracle import tangent
    sc = _turning_column() if case == "column" else _translating_periodic()
    n = len(sc.particles)
    rng = np.random.default_rng(3)
    w = rng.standard_normal((n, 3))
    u = rng.standard_normal((n, 3)) * 1e-3
    dirs = [rng.standard_normal((n, 3)) for _ in range(3)]
    s = fundem.Simulation.from_scenario(sc, records=False)
    s.detect()
    s.adjoint_begin(max(steps // 4, 1))
    s.adjoint_forward(steps)
    gv0, gp = s.adjoint_backward(w, u)
    st = s.state()
    s.adjoint_end()
    s.close()

    tr = tangent.TangentRun(sc, dirs)
    tr.step(steps)
    ref = tr.directional(w, u)
    so = tr.o.state()
    tr.close()
    assert np.abs(st["pos"] - so["pos"]).max() <= 1e-12 * np.abs(so["pos"]).max()
    got = np.concatenate([gp.ravel(), [float(np.sum(gv0 * d)) for d in dirs]])
    assert got.shape == ref.shape
    scale = np.abs(ref).max()
    for k in range(len(ref)):
        assert abs(got[k] - ref[k]) <= 1e-6 * abs(ref[k]) + 1e-9 * scale, (k, got[k], ref[k])
