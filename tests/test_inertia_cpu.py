"""The two inverse-inertia rules, on the CPU oracle.

The reference's inverse() (myMat.h:163-194) returns the zero matrix when
|det I| < 1e-30, so the mm-scale bodies of the pour never change their
angular velocity.  The physical rule inverts every inertia that is not
singular relative to its own scale (|det I| > 1e-12 max|I_ii|^3)."""
import dataclasses

import numpy as np
import pytest

import parity_cases as PC


def _sym(v):
    xx, yy, zz, xy, xz, yz = v
    return np.array([[xx, xy, xz], [xy, yy, yz], [xz, yz, zz]])


def _world(oracle_mod, inertia):
    sc = dataclasses.replace(PC.pour_mm(), inertia=inertia)
    return sc, oracle_mod.OracleWorld.from_scenario(sc)


def test_reference_rule_zeroes_mm_inertia(oracle_mod):
    sc, o = _world(oracle_mod, "reference")
    for k in range(len(sc.particle_geometries)):
        g = o.geometry(k)
        assert np.linalg.det(_sym(g["inertia"])) < 1e-30
        assert not np.any(g["inv_inertia"])


def test_physical_rule_inverts_mm_inertia(oracle_mod):
    sc, o = _world(oracle_mod, "physical")
    for k in range(len(sc.particle_geometries)):
        g = o.geometry(k)
        I = _sym(g["inertia"])
        Ii = _sym(g["inv_inertia"])
        assert np.abs(Ii @ I - np.eye(3)).max() < 1e-12
    # walls keep zero inertia and zero inverse under either rule
    w = o.geometry(0, wall=True)
    assert not np.any(w["inv_inertia"])


def test_physical_rule_zeroes_relatively_singular_inertia(oracle_mod):
    """A body with no extent along one axis (a rod or a point) stays
    non-rotating under the physical rule."""
    sc = dataclasses.replace(PC.pour_mm(), inertia="physical")
    geos = list(sc.particle_geometries)
    rod = dataclasses.replace(geos[0], density=None, mass=1e-5, inertia=np.array([4e-12, 4e-12, 0.0, 0.0, 0.0, 0.0]))
    near = dataclasses.replace(geos[1], density=None, mass=1e-5,
                               inertia=np.array([4e-12, 4e-12, 4e-24, 0.0, 0.0, 0.0]))
    sc = dataclasses.replace(sc, particle_geometries=[rod, near] + geos[2:])
    o = oracle_mod.OracleWorld.from_scenario(sc)
    assert not np.any(o.geometry(0)["inv_inertia"])
    assert not np.any(o.geometry(1)["inv_inertia"])
    assert np.any(o.geometry(2)["inv_inertia"])


def test_mode_switch_recomputes_existing_geometries(oracle_mod):
    sc, o = _world(oracle_mod, "reference")
    o.L.orc_set_inertia_mode(o.w, 1)
    assert np.any(o.geometry(0)["inv_inertia"])
    o.L.orc_set_inertia_mode(o.w, 0)
    assert not np.any(o.geometry(0)["inv_inertia"])


@pytest.mark.parametrize("inertia", ["reference", "physical"])
def test_mm_bodies_turn_only_under_the_physical_rule(oracle_mod, inertia):
    sc, o = _world(oracle_mod, inertia)
    o.initial_detect()
    w0 = o.state()["angvel"].copy()
    o.step(20)
    st = o.state()
    touched = np.abs(st["torque"]).max(axis=1) > 0.0
    assert touched.sum() > 0
    if inertia == "reference":
        assert np.array_equal(st["angvel"], w0)
    else:
        assert np.abs(st["angvel"][touched] - w0[touched]).max() > 0.0
        # the quaternions stay unit
        assert np.abs(np.linalg.norm(st["quat"], axis=1) - 1.0).max() < 1e-12


def test_free_tumbling_body_keeps_its_angular_momentum(oracle_mod):
    """Known answer for the physical rule: a free mm-scale superellipsoid
    (no gravity, no contacts) spinning about no principal axis tumbles
    (its angular velocity changes) while its world-frame angular momentum
    R I R^T w stays fixed to the integrator's first-order error; under the
    reference rule it keeps its angular velocity exactly."""
    base = PC.pour_mm()

    def run(inertia, steps=2000):
        sc = dataclasses.replace(base, inertia=inertia, gravity=np.zeros(3), walls=type(base.walls).empty(),
                                 wall_geometries=[], dt=1e-6)
        P = sc.particles
        keep = slice(0, 1)
        sc = dataclasses.replace(sc, particles=type(P)(P.pos[keep].copy(), np.zeros((1, 3)),
                                                     np.array([[300.0, -120.0, 200.0]]), P.quat[keep].copy(),
                                                     P.mat[keep].copy(), P.geo[keep].copy()))
        o = oracle_mod.OracleWorld.from_scenario(sc)
        I = o.geometry(int(sc.particles.geo[0]))["inertia"]
        o.initial_detect()
        w0 = o.state()["angvel"][0].copy()
        L = []
        for _ in range(4):
            st = o.state()
            L.append(_world_momentum(I, st["quat"][0], st["angvel"][0]))
            o.step(steps // 4)
        st = o.state()
        L.append(_world_momentum(I, st["quat"][0], st["angvel"][0]))
        o.close()
        return w0, st["angvel"][0], np.array(L)

    w0, w1, L = run("physical")
    assert np.linalg.norm(w1 - w0) > 1e-2 * np.linalg.norm(w0)       # it tumbles (2% here)
    drift = np.abs(L - L[0]).max() / np.linalg.norm(L[0])
    assert drift < 1e-5, drift                                         # observed 3.5e-7
    w0, w1, _ = run("reference")
    assert np.array_equal(w0, w1)


def _world_momentum(I6, q, w):
    q0, q1, q2, q3 = q
    R = np.array([[1 - 2 * (q2 * q2 + q3 * q3), 2 * (q1 * q2 - q0 * q3), 2 * (q1 * q3 + q0 * q2)],
                  [2 * (q1 * q2 + q0 * q3), 1 - 2 * (q1 * q1 + q3 * q3), 2 * (q2 * q3 - q0 * q1)],
                  [2 * (q1 * q3 - q0 * q2), 2 * (q2 * q3 + q0 * q1), 1 - 2 * (q1 * q1 + q2 * q2)]])
    return R @ _sym(I6) @ R.T @ w
