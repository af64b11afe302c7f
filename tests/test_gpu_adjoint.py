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
    sim, sc, info = workloads.bonded_column(n=512, footprint=(8, 8), seed=request.param, settle_steps=0)
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


def test_adjoint_refuses_turning_bodies_with_bonds(fundem):
    import parity_cases
    from fundem_b200 import scenario as S
    sc = parity_cases.cluster()  # cm bodies: nonzero inverse inertia
    p = sc.particles.pos
    sc.bonds = S.Bonds(np.array([0], np.int32), np.array([1], np.int32), 0.5 * (p[0:1] + p[1:2]),
                       np.array([[1.0, 0.0, 0.0]]), np.array([1e-3]), np.array([np.linalg.norm(p[0] - p[1])]),
                       np.array([1e8]), np.array([0.3]), np.array([1e6]), np.array([0.0]), np.array([0.0]))
    s = fundem.Simulation.from_scenario(sc)
    s.detect()
    with pytest.raises(fundem.FundemError):
        s.adjoint_begin(10)
    s.close()


def _cluster_loss(fundem, sc, w, u, y, z, steps):
    s = fundem.Simulation.from_scenario(sc, records=False)
    s.detect()
    s.step(steps)
    s.sync()
    st = s.state()
    s.close()
    return float(np.sum(w * st["pos"]) + np.sum(u * st["vel"]) + np.sum(y * st["quat"]) + np.sum(z * st["angvel"]))


def test_turning_adjoint_matches_finite_differences(fundem):
    """Turning cm-scale bodies (the cluster case: angular velocities of about
    20 rad/s, five walls, friction, two materials), 10 steps in three
    checkpoint segments: the adjoint's gradients with respect to both
    materials' kn, ks, damping ratio and friction coefficient, initial
    velocities and initial angular velocities against central finite
    differences (relative step 1e-4 for the parameters, 1e-5 m/s and 1e-4
    rad/s for the initial state), through the world-frame inertia of the
    kicks, the normalised quaternion step and the torques' lever arms.
    Loss: L = sum(w x_T) + sum(u v_T) + sum(y q_T) + sum(z w_T)."""
    import copy
    import parity_cases
    steps, K = 10, 4
    sc = parity_cases.cluster()
    n = len(sc.particles)
    rng = np.random.default_rng(21)
    w = rng.standard_normal((n, 3))
    u = rng.standard_normal((n, 3)) * 1e-2
    y = rng.standard_normal((n, 4)) * 1e-2
    z = rng.standard_normal((n, 3)) * 1e-4
    s = fundem.Simulation.from_scenario(sc, records=False)
    s.detect()
    s.adjoint_begin(K)
    s.adjoint_forward(steps)
    gv0, gw0, gp = s.adjoint_backward_rot(w, u, y, z)
    s.adjoint_end()
    s.close()
    assert np.all(np.isfinite(gw0)) and np.abs(gw0).max() > 0
    L0 = _cluster_loss(fundem, sc, w, u, y, z, steps)

    def with_material(mi, k, scale):
        s2 = copy.deepcopy(sc)
        m = list(s2.particle_materials[mi])
        if k == 2:  # damping ratio: perturb through the restitution the API takes
            zeta = _zeta(m[3]) * scale
            m[3] = float(np.exp(-np.pi * zeta / np.sqrt(1.0 - zeta * zeta)))
        else:
            m[[0, 1, None, 2][k]] *= scale
        s2.particle_materials[mi] = tuple(m)
        return s2

    h = 1e-4
    for mi in range(2):
        m = sc.particle_materials[mi]
        base = [m[0], m[1], _zeta(m[3]), m[2]]
        for k in range(4):
            Lp = _cluster_loss(fundem, with_material(mi, k, 1 + h), w, u, y, z, steps)
            Lm = _cluster_loss(fundem, with_material(mi, k, 1 - h), w, u, y, z, steps)
            _check_fd(f"material {mi} param {k}", gp[mi, k] * base[k], L0, Lp, Lm, h,
                      atol=1e-9 * max(abs(L0), 1.0))
    for name, grad, key, step in (("v0", gv0, "vel", 1e-5), ("w0", gw0, "angvel", 1e-4)):
        for _ in range(3):
            i, c = int(rng.integers(0, n - 1)), int(rng.integers(0, 3))
            sp, sm = copy.deepcopy(sc), copy.deepcopy(sc)
            getattr(sp.particles, key)[i, c] += step
            getattr(sm.particles, key)[i, c] -= step
            Lp = _cluster_loss(fundem, sp, w, u, y, z, steps)
            Lm = _cluster_loss(fundem, sm, w, u, y, z, steps)
            _check_fd(f"{name}[{i},{c}]", grad[i, c] * step, L0, Lp, Lm, step / step,
                      atol=1e-9 * max(abs(L0), 1.0))


def test_checkpoint_interval_autotuner(fundem):
    """The autotuner times forward + backward for several checkpoint
    intervals and picks one; the gradients do not depend on the interval,
    since each segment's re-run repeats the forward run (they agree to
    rounding: the reverse sweep adds to particles with atomics)."""
    from fundem_b200 import autotune, workloads
    sim, sc, info = workloads.bonded_column(n=512, footprint=(8, 8), seed=11, settle_steps=0)
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
    sim, sc, info = workloads.bonded_column(n=512, footprint=(8, 8), seed=12, settle_steps=0)
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


def test_turning_adjoint_matches_tangent_reference(fundem, oracle_mod):
    """The reverse sweep of turning bodies (fundem_adjoint_backward_rot)
    against the FP64 CPU forward-mode reference along the oracle's own run
    (oracle/tangent.py with orientations, angular velocities and torques):
    the rotating cluster (cm bodies at about 20 rad/s, two materials, five
    walls), 10 steps in three checkpoint segments, a loss on final
    positions, velocities, orientations and angular velocities.  Both
    materials' four gradients and the projections of d L / d v_0 and
    d L / d w_0 on random directions agree to 1e-5 relative (observed
    1.2e-6 at most, on the damping ratio: the step takes the damping
    coefficients' square roots in single precision, as the reference does,
    and the tangent reference evaluates the law's values in double)."""
    import parity_cases
    from oracle import tangent
    steps, K = 10, 4
    sc = parity_cases.cluster()
    n = len(sc.particles)
    rng = np.random.default_rng(31)
    w = rng.standard_normal((n, 3))
    u = rng.standard_normal((n, 3)) * 1e-2
    y = rng.standard_normal((n, 4)) * 1e-2
    z = rng.standard_normal((n, 3)) * 1e-4
    vdirs = [rng.standard_normal((n, 3)) for _ in range(2)]
    wdirs = [rng.standard_normal((n, 3)) for _ in range(2)]
    s = fundem.Simulation.from_scenario(sc, records=False)
    s.detect()
    s.adjoint_begin(K)
    s.adjoint_forward(steps)
    gv0, gw0, gp = s.adjoint_backward_rot(w, u, y, z)
    st = s.state()
    s.adjoint_end()
    s.close()

    tr = tangent.TangentRun(sc, vdirs, wdirs)
    assert tr.turning
    tr.step(steps)
    ref = tr.directional(w, u, y, z)
    so = tr.o.state()
    tr.close()
    assert np.abs(st["pos"] - so["pos"]).max() <= 1e-12 * np.abs(so["pos"]).max()
    got = np.concatenate([gp.ravel(), [float(np.sum(gv0 * d)) for d in vdirs],
                          [float(np.sum(gw0 * d)) for d in wdirs]])
    assert got.shape == ref.shape
    scale = np.abs(ref).max()
    print("turning adjoint vs tangent reference, relative:", np.abs(got - ref) / (np.abs(ref) + 1e-9 * scale))
    for k in range(len(ref)):
        assert abs(got[k] - ref[k]) <= 1e-5 * abs(ref[k]) + 1e-9 * scale, (k, got[k], ref[k])


def test_mixed_precision_adjoint(fundem, oracle_mod):
    """The adjoint of the FP32_MIXED step (its recorded single-precision run
    swept with double-precision Jacobians) against the FP64 reference
    derivative and against the FP64 adjoint: within 1e-3 relative (observed
    6e-5 with single-precision Jacobians).

    Central differences of the mixed forward run cannot check it at this
    size: single-precision forces put a rounding staircase into the loss
    that is comparable to the loss change of a 1e-3 parameter step (the
    forward and backward differences of kn differ by 13% there)."""
    from oracle import tangent
    from fundem_b200 import workloads
    sim, sc, info = workloads.bonded_column(n=512, footprint=(8, 8), seed=11, settle_steps=0)
    sim.close()
    sc.wall_materials = [(0.7, 0.9)]
    n = len(sc.particles)
    rng = np.random.default_rng(7)
    w = rng.standard_normal((n, 3))
    u = rng.standard_normal((n, 3)) * 1e-3
    dirs = [rng.standard_normal((n, 3)) for _ in range(2)]

    def grads(precision, probe=False):
        s = fundem.Simulation.from_scenario(sc, records=False)
        s.set_precision(precision)
        s.detect()
        s.adjoint_begin(K)
        s.adjoint_forward(T)
        if probe:  # the precision may not change while recording
            s.set_precision(fundem.FP64 if precision == fundem.FP32_MIXED else fundem.FP32_MIXED)
            with pytest.raises(fundem.FundemError):
                s.adjoint_forward(1)
            s.set_precision(precision)
        gv0, gp = s.adjoint_backward(w, u)
        s.adjoint_end()
        s.close()
        return np.concatenate([gp.ravel(), [float(np.sum(gv0 * d)) for d in dirs]])

    got = grads(fundem.FP32_MIXED, probe=True)
    g64 = grads(fundem.FP64)
    tr = tangent.TangentRun(sc, dirs)
    tr.step(T)
    ref = tr.directional(w, u)
    tr.close()
    scale = np.abs(ref).max()
    dev = np.abs(got - ref) / (np.abs(ref) + 1e-6 * scale)
    dev64 = np.abs(got - g64) / (np.abs(g64) + 1e-6 * scale)
    print("mixed adjoint vs FP64 reference derivative, relative:", dev)
    print("mixed adjoint vs FP64 adjoint, relative:", dev64)
    assert dev.max() < 1e-3, (got, ref)
    assert dev64.max() < 1e-3, (got, g64)


def test_mixed_adjoint_on_the_pour(fundem):
    """The adjoint pour (4,096 particles in a box of six walls, 100 steps, in
    which wall contacts separate) gives finite mixed-precision gradients:
    the material gradients follow the FP64 ones within 1e-3 relative, the
    initial-velocity gradients within 1e-2 normwise.  Single-precision
    Jacobians gave non-finite gradients here."""
    from fundem_b200 import workloads
    sim, sc = workloads.adjoint_pour(n=4096)
    sim.close()
    n = len(sc.particles)
    dl = np.zeros((n, 3))
    dl[:, 2] = 1.0 / n
    out = []
    for precision in (fundem.FP64, fundem.FP32_MIXED):
        s = fundem.Simulation.from_scenario(sc, records=False)
        s.set_precision(precision)
        s.detect()
        s.adjoint_begin(50)
        s.adjoint_forward(100)
        gv0, gp = s.adjoint_backward(dl, np.zeros((n, 3)))
        s.adjoint_end()
        s.close()
        assert np.isfinite(gv0).all() and np.isfinite(gp).all()
        out.append((gv0, gp))
    (v64, p64), (v32, p32) = out
    assert np.all(np.abs(p32 - p64) <= 1e-3 * np.abs(p64) + 1e-6 * np.abs(p64).max())
    # per particle the two runs can differ in a contact's first step, which
    # moves that particle's gradient (up to 0.75% of the largest entry here);
    # over all particles they agree closely
    assert np.linalg.norm(v32 - v64) <= 1e-2 * np.linalg.norm(v64)
