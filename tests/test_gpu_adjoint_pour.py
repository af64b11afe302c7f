"""Config 3's adjoint on its own workload, 16 seeds.

The pour (4,096 superellipsoids from 2 templates, a box of six plane walls,
dt = 1e-6 s) is poured into a bed first (the library's own steps at 5e-6 s,
untimed, until the kinetic energy falls below 1e-3 of the fall's peak or
40,000 steps), so the checked window is full of particle and wall
contacts.  Over the next 100 steps (checkpoints every 25) the loss of config
3 -- the packing fraction, N V / (A H) with H twice the mean particle height,
plus the mean-square displacement of 64 tagged particles -- is
differentiated with respect to the particle material's kn, ks, damping ratio
and friction coefficient (relative step 1e-4) and to two initial velocity
components (1e-5 m/s), and compared with central finite differences of the
GPU forward run to 1e-3 relative (one-sided where a contact event falls
inside the step, as in test_gpu_adjoint.py), with an absolute floor of 1e-3
of the seed's largest gradient of the group: in a bed at rest some
gradients (the damping ratio's, typically) are a thousandth of the others,
and the loss changes they cause are the size of the contact events' jumps.
The FP32_MIXED adjoint of the same window agrees with the FP64 adjoint to
1e-2 on the material gradients.
"""
import copy

import numpy as np
import pytest

from test_gpu_adjoint import _check_fd, _zeta

pytestmark = pytest.mark.gpu

T, K, SEEDS = 100, 25, 16


def _bed(fundem, seed):
    from fundem_b200 import workloads
    sim, sc = workloads.adjoint_pour(n=4096, seed=seed, settle_steps=40000)
    sim.close()
    return sc


def _geometry(sc):
    masses = np.array([g.mass for g in sc.particle_geometries])[sc.particles.geo]
    vol = float(np.sum(masses) / 2500.0)
    lo, hi = sc.walls.pos.min(axis=0), sc.walls.pos.max(axis=0)
    return vol, float((hi[0] - lo[0]) * (hi[1] - lo[1])), float(lo[2])


def _loss_and_grad(sc, pos):
    vol, area, z0 = _geometry(sc)
    n = len(pos)
    tag = np.arange(0, n, n // 64)[:64]
    x0 = sc.particles.pos
    H = 2.0 * float(np.mean(pos[:, 2] - z0))
    phi = vol / (area * H)
    d = pos[tag] - x0[tag]
    L = phi + float(np.mean(np.sum(d * d, axis=1)))
    g = np.zeros((n, 3))
    g[:, 2] = -phi / H * 2.0 / n
    g[tag] += 2.0 * d / len(tag)
    return L, g


def _forward_loss(fundem, sc):
    s = fundem.Simulation.from_scenario(sc, records=False)
    s.detect()
    s.step(T)
    s.sync()
    pos = s.state()["pos"]
    s.close()
    return _loss_and_grad(sc, pos)[0]


def _adjoint(fundem, sc, precision):
    s = fundem.Simulation.from_scenario(sc, records=False)
    s.set_precision(precision)
    s.detect()
    s.adjoint_begin(K)
    s.adjoint_forward(T)
    st = s.state()
    contacts = s.num_contacts(fundem.PP) + s.num_contacts(fundem.PW)
    L, g = _loss_and_grad(sc, st["pos"])
    gv0, gp = s.adjoint_backward(g, np.zeros_like(g))
    s.adjoint_end()
    s.close()
    return L, gv0, gp[0], contacts


def _with(sc, k, scale):
    s2 = copy.deepcopy(sc)
    kn, ks, mu, e = s2.particle_materials[0]
    if k == 0:
        kn *= scale
    elif k == 1:
        ks *= scale
    elif k == 2:
        z = _zeta(e) * scale
        e = float(np.exp(-np.pi * z / np.sqrt(1.0 - z * z)))
    else:
        mu *= scale
    s2.particle_materials[0] = (kn, ks, mu, e)
    return s2


def test_pour_adjoint_16_seeds(fundem):
    h = 1e-4
    for seed in range(SEEDS):
        sc = _bed(fundem, seed)
        L0, gv0, gp, contacts = _adjoint(fundem, sc, fundem.FP64)
        assert contacts > 2500, (seed, contacts)   # a bed: thousands of node contacts
        assert abs(_forward_loss(fundem, sc) - L0) <= 1e-12 * abs(L0)
        kn, ks, mu, e = sc.particle_materials[0]
        base = [kn, ks, _zeta(e), mu]
        g = [gp[k] * base[k] for k in range(4)]
        floor = 1e-9 * abs(L0) + 1e-3 * max(abs(x) for x in g)
        for k in range(4):
            Lp = _forward_loss(fundem, _with(sc, k, 1 + h))
            Lm = _forward_loss(fundem, _with(sc, k, 1 - h))
            _check_fd(f"seed {seed} param {k}", g[k], L0, Lp, Lm, h, atol=floor)
        rng = np.random.default_rng(seed)
        picks = [(int(rng.integers(0, len(sc.particles))), int(rng.integers(0, 3))) for _ in range(2)]
        dv = 1e-5
        floor = 1e-9 * abs(L0) + 1e-3 * max(abs(gv0[i, c] * dv) for i, c in picks)
        for i, c in picks:
            sp, sm = copy.deepcopy(sc), copy.deepcopy(sc)
            sp.particles.vel[i, c] += dv
            sm.particles.vel[i, c] -= dv
            _check_fd(f"seed {seed} v0[{i},{c}]", gv0[i, c] * dv, L0, _forward_loss(fundem, sp),
                      _forward_loss(fundem, sm), 1.0, atol=floor)
        print(f"seed {seed}: {contacts} node contacts, d L / d log(kn, ks, zeta, mu) = {g}")
        # the mixed-precision adjoint of the same window
        _, _, gp32, _ = _adjoint(fundem, sc, fundem.FP32_MIXED)
        scale = np.abs(gp * np.array(base)).max()
        assert np.abs((gp32 - gp) * np.array(base)).max() <= 1e-2 * scale, (seed, gp, gp32)
