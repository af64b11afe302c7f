"""The tangent-linear reference (oracle/tangent.py) against central finite
differences of the oracle.

The tangent reference is the FP64 CPU check of the GPU adjoint, so it is
pinned here first.  The finite differences run the oracle with its damping
square roots in double precision (orc_set_damping_sqrt64): the reference's
single-precision roots make the loss a staircase at the 1e-8 level in kn,
ks and the damping ratio, which steps of 1e-6 cannot resolve.  With smooth
damping, central differences with a relative step of 1e-6 agree with the
tangent to 1e-6 relative (observed 1e-8) over 20 steps of:

* the periodic bonded case with its inertia zeroed (translating bodies that
  keep a constant angular velocity of about 10 rad/s): particle pairs, two
  walls with one moving, x/y ghosts and bonds;
* the mm-scale pour in its box of walls.
"""
import copy

import numpy as np
import pytest

import parity_cases as PC

T = 20


def _translating(sc):
    sc = copy.deepcopy(sc)
    for g in sc.particle_geometries:
        assert g.density is None
        g.inertia = np.zeros(6)
    # walls with more friction and restitution than the particles, away from
    # the kink of min(...)
    sc.wall_materials = [(0.7, 0.9)] * len(sc.wall_materials)
    return sc


def _zeta(e):
    lr = np.log(e)
    return -lr / np.sqrt(lr * lr + np.pi * np.pi)


def _with(sc, name=None, x=None, dv=None):
    s2 = copy.deepcopy(sc)
    kn, ks, mu, e = s2.particle_materials[0]
    if name == "kn":
        kn = x
    elif name == "ks":
        ks = x
    elif name == "mu":
        mu = x
    elif name == "zeta":
        e = float(np.exp(-np.pi * x / np.sqrt(1.0 - x * x)))
    s2.particle_materials[0] = (kn, ks, mu, e)
    if dv is not None:
        s2.particles.vel = s2.particles.vel + dv
    return s2


@pytest.fixture
def smooth_damping(oracle_mod):
    L = oracle_mod.lib()
    L.orc_set_damping_sqrt64(1)
    yield
    L.orc_set_damping_sqrt64(0)


@pytest.mark.parametrize("case", ["periodic", "pour_mm"])
def test_tangent_matches_central_differences(oracle_mod, smooth_damping, case):
    from oracle import tangent
    sc = PC.CASES[case]()
    sc = _translating(sc) if case == "periodic" else copy.deepcopy(sc)
    if case == "pour_mm":
        sc.wall_materials = [(0.7, 0.9)] * len(sc.wall_materials)
    n = len(sc.particles)
    rng = np.random.default_rng(1)
    w = rng.standard_normal((n, 3))
    u = rng.standard_normal((n, 3)) * 1e-3
    r = rng.standard_normal((n, 3))
    tr = tangent.TangentRun(sc, [r])
    tr.step(T)
    D = tr.directional(w, u)
    assert tr.max_overlap_dev < 1e-9 and tr.max_spring_dev < 1e-9
    tr.close()

    def loss(s2):
        o = oracle_mod.OracleWorld.from_scenario(s2)
        o.initial_detect()
        o.step(T)
        st = o.state()
        o.close()
        return float(np.sum(w * st["pos"]) + np.sum(u * st["vel"]))

    L0 = loss(sc)
    kn0, ks0, mu0, e0 = sc.particle_materials[0]
    cases = [("kn", kn0, 0), ("ks", ks0, 1), ("zeta", _zeta(e0), 2), ("mu", mu0, 3)]
    for name, x0, k in cases:
        h = 1e-6 * x0
        Lp, Lm = loss(_with(sc, name, x0 + h)), loss(_with(sc, name, x0 - h))
        central, fwd, bwd = (Lp - Lm) / (2 * h), (Lp - L0) / h, (L0 - Lm) / h
        atol = 1e-9 * max(abs(L0), 1.0) / h
        if abs(fwd - bwd) <= 1e-3 * abs(central) + atol:
            assert abs(D[k] - central) <= 1e-6 * abs(central) + atol, (name, D[k], central)
        else:  # a contact event inside [x - h, x + h]: one side is smooth
            assert min(abs(D[k] - fwd), abs(D[k] - bwd)) <= 1e-4 * abs(D[k]) + atol, (name, D[k], fwd, bwd)
    h = 1e-6
    Lp, Lm = loss(_with(sc, dv=h * r)), loss(_with(sc, dv=-h * r))
    central = (Lp - Lm) / (2 * h)
    assert abs(D[4] - central) <= 1e-6 * abs(central) + 1e-9, (D[4], central)


def test_tangent_two_materials(oracle_mod, smooth_damping):
    """The 48-body cluster with two particle materials (harmonic-mean
    stiffness and minimum friction and restitution between them), five
    walls and bodies spinning at about 20 rad/s, made translating: all eight
    material gradients against central differences (relative step 1e-6)
    within 1e-4 relative (observed 2e-5 at most, on the smallest ones)."""
    from oracle import tangent
    sc = copy.deepcopy(PC.cluster())
    for g in sc.particle_geometries:
        if g.density is not None:  # the template registered through a density
            g.density = None
            g.mass = 1.5e-3
        g.inertia = np.zeros(6)
    sc.wall_materials = [(0.9, 0.95)] * len(sc.wall_materials)
    assert len(sc.particle_materials) == 2 and set(np.unique(sc.particles.mat)) == {0, 1}
    n = len(sc.particles)
    rng = np.random.default_rng(2)
    w = rng.standard_normal((n, 3))
    u = rng.standard_normal((n, 3)) * 1e-3
    tr = tangent.TangentRun(sc)
    tr.step(T)
    D = tr.directional(w, u)
    tr.close()

    def loss(s2):
        o = oracle_mod.OracleWorld.from_scenario(s2)
        o.initial_detect()
        o.step(T)
        st = o.state()
        o.close()
        return float(np.sum(w * st["pos"]) + np.sum(u * st["vel"]))

    for m in range(2):
        kn, ks, mu, e = sc.particle_materials[m]
        for k, x0 in enumerate((kn, ks, _zeta(e), mu)):
            def moved(x):
                s2 = copy.deepcopy(sc)
                a = list(s2.particle_materials[m])
                if k == 2:
                    a[3] = float(np.exp(-np.pi * x / np.sqrt(1.0 - x * x)))
                else:
                    a[(0, 1, None, 2)[k]] = x
                s2.particle_materials[m] = tuple(a)
                return s2
            h = 1e-6 * x0
            central = (loss(moved(x0 + h)) - loss(moved(x0 - h))) / (2 * h)
            assert abs(D[4 * m + k] - central) <= 1e-4 * abs(central), (m, k, D[4 * m + k], central)


def test_tangent_turning_bodies(oracle_mod, smooth_damping):
    """The 48-body cluster as it is -- cm bodies that turn (angular
    velocities of about 20 rad/s, nonzero inverse inertia), two materials,
    five walls -- over 10 steps: the derivatives through the world-frame
    inertia of the kicks, the normalised quaternion step and the torques'
    lever arms, of a loss on final positions, velocities, orientations and
    angular velocities, against central differences of the oracle: the eight
    material gradients (relative step 1e-6) and initial velocity and angular
    velocity directions (steps 1e-6 m/s and 1e-5 rad/s) to 1e-4 relative
    (observed 1.1e-7 at most)."""
    from oracle import tangent
    sc = copy.deepcopy(PC.cluster())
    steps = 10
    n = len(sc.particles)
    rng = np.random.default_rng(6)
    w = rng.standard_normal((n, 3))
    u = rng.standard_normal((n, 3)) * 1e-2
    y = rng.standard_normal((n, 4)) * 1e-2
    z = rng.standard_normal((n, 3)) * 1e-4
    rv, rw = rng.standard_normal((n, 3)), rng.standard_normal((n, 3))
    tr = tangent.TangentRun(sc, [rv], [rw])
    assert tr.turning
    tr.step(steps)
    D = tr.directional(w, u, y, z)
    assert tr.max_quat_dev < 1e-14 and tr.max_overlap_dev < 1e-9 and tr.max_spring_dev < 1e-9
    assert np.abs(tr.dw).max() > 0 and np.abs(tr.dq).max() > 0
    tr.close()

    def loss(s2):
        o = oracle_mod.OracleWorld.from_scenario(s2)
        o.initial_detect()
        o.step(steps)
        st = o.state()
        o.close()
        return float(np.sum(w * st["pos"]) + np.sum(u * st["vel"]) + np.sum(y * st["quat"])
                     + np.sum(z * st["angvel"]))

    L0 = loss(sc)
    for m in range(2):
        kn, ks, mu, e = sc.particle_materials[m]
        for k, x0 in enumerate((kn, ks, _zeta(e), mu)):
            def moved(x):
                s2 = copy.deepcopy(sc)
                a = list(s2.particle_materials[m])
                if k == 2:
                    a[3] = float(np.exp(-np.pi * x / np.sqrt(1.0 - x * x)))
                else:
                    a[(0, 1, None, 2)[k]] = x
                s2.particle_materials[m] = tuple(a)
                return s2
            h = 1e-6 * x0
            Lp, Lm = loss(moved(x0 + h)), loss(moved(x0 - h))
            central, fwd, bwd = (Lp - Lm) / (2 * h), (Lp - L0) / h, (L0 - Lm) / h
            atol = 1e-9 * max(abs(L0), 1.0) / h
            if abs(fwd - bwd) <= 1e-3 * abs(central) + atol:
                assert abs(D[4 * m + k] - central) <= 1e-4 * abs(central) + atol, (m, k, D[4 * m + k], central)
            else:  # a contact event inside [x - h, x + h]: one side is smooth
                assert min(abs(D[4 * m + k] - fwd), abs(D[4 * m + k] - bwd)) <= 1e-4 * abs(D[4 * m + k]) + atol, \
                    (m, k, D[4 * m + k], fwd, bwd)
    for idx, key, r, h in ((8, "vel", rv, 1e-6), (9, "angvel", rw, 1e-5)):
        sp, sm = copy.deepcopy(sc), copy.deepcopy(sc)
        setattr(sp.particles, key, getattr(sc.particles, key) + h * r)
        setattr(sm.particles, key, getattr(sc.particles, key) - h * r)
        central = (loss(sp) - loss(sm)) / (2 * h)
        assert abs(D[idx] - central) <= 1e-4 * abs(central) + 1e-9, (key, D[idx], central)


@pytest.mark.parametrize("case", ["periodic", "cluster"])
def test_reverse_reference_adjoint_matches_tangent(oracle_mod, case):
    """The reverse-mode reference adjoint (oracle/reverse.py: the whole run
    recorded, one backward sweep giving every initial-velocity gradient and
    every material gradient) against the forward-mode reference derivative:
    the material gradients and the projections of d L / d v_0 on random
    directions agree to 1e-12 relative (observed 2e-14), the dot-product
    test of an adjoint.  Periodic bonded case with ghosts and the
    two-material cluster, both translating, 30 steps."""
    from oracle import reverse, tangent
    sc = copy.deepcopy(PC.CASES[case]())
    for g in sc.particle_geometries:
        if g.density is not None:
            g.density = None
            g.mass = 1.5e-3
        g.inertia = np.zeros(6)
    sc.wall_materials = [(0.9, 0.95)] * len(sc.wall_materials)
    n = len(sc.particles)
    rng = np.random.default_rng(4)
    w = rng.standard_normal((n, 3))
    u = rng.standard_normal((n, 3)) * 1e-3
    dirs = [rng.standard_normal((n, 3)) for _ in range(2)]
    tr = tangent.TangentRun(sc, dirs)
    tr.step(30)
    ref = tr.directional(w, u)
    tr.close()
    rr = reverse.ReverseRun(sc)
    rr.step(30)
    gv0, gp = rr.gradients(w, u)
    rr.close()
    got = np.concatenate([gp.ravel(), [float(np.sum(gv0 * d)) for d in dirs]])
    assert np.all(np.abs(got - ref) <= 1e-12 * np.abs(ref) + 1e-15 * np.abs(ref).max()), (got, ref)


def test_autograd_wrapper_with_the_reference_adjoint(oracle_mod):
    """The torch.autograd wrapper of the adjoint (tests/adjoint_autograd.py)
    over the CPU reference adjoint: a loss that is nonlinear in the final
    state (mean height plus the kinetic-energy-like sum of squared final
    velocities) differentiated by loss.backward() gives the material and
    initial-velocity gradients of the forward-mode derivative along the
    same directions."""
    import torch
    from oracle import tangent
    import adjoint_autograd as AG
    sc = copy.deepcopy(PC.periodic())
    for g in sc.particle_geometries:
        g.inertia = np.zeros(6)
    sc.wall_materials = [(0.9, 0.95)]
    n, steps = len(sc.particles), 20
    v0 = torch.tensor(sc.particles.vel, dtype=torch.float64, requires_grad=True)
    params = torch.tensor(AG.material_parameters(sc), dtype=torch.float64, requires_grad=True)
    x, v = AG.DEMRun.apply(v0, params, AG.OracleBackend(sc), steps)
    loss = x[:, 2].mean() + 1e-2 * (v * v).sum()
    loss.backward()
    # the same derivative, direction by direction, with the loss gradient at
    # the final state
    rng = np.random.default_rng(9)
    r = rng.standard_normal((n, 3))
    tr = tangent.TangentRun(sc, [r])
    tr.step(steps)
    st = tr.o.state()
    dl_dx = np.zeros((n, 3))
    dl_dx[:, 2] = 1.0 / n
    D = tr.directional(dl_dx, 2e-2 * st["vel"])
    tr.close()
    got = np.concatenate([params.grad.numpy().ravel(), [float(np.sum(v0.grad.numpy() * r))]])
    # same run (the restitution coefficient passes through the damping ratio)
    assert np.abs(st["pos"] - x.detach().numpy()).max() <= 1e-14 * np.abs(st["pos"]).max()
    assert np.all(np.abs(got - D) <= 1e-10 * np.abs(D) + 1e-14 * np.abs(D).max()), (got, D)


def test_reference_derivatives_refuse_what_they_do_not_differentiate():
    """Bonds between turning bodies and sector images are outside the
    frozen-topology model the tangent reference (and the GPU adjoint)
    differentiates; the reverse reference differentiates translating bodies
    only."""
    from oracle import reverse, tangent
    with pytest.raises(AssertionError):
        tangent.TangentRun(PC.periodic())          # cm bodies with bonds
    with pytest.raises(AssertionError):
        reverse.ReverseRun(PC.cluster())           # turning bodies
    sc = copy.deepcopy(PC.sector())
    for g in sc.particle_geometries:
        g.inertia = np.zeros(6)
    with pytest.raises(AssertionError):
        reverse.ReverseRun(sc)
