"""Mixed-precision mode (FUNDEM_FP32_MIXED) against FP64 on the GPU.

The mode evaluates the SDF interpolation and gradient, the contact and bond
laws and the force sums in single precision, and keeps positions,
orientations, the rigid transforms, their integration and the spring history
in double precision.

Gate, after 1,000 steps: norm-wise relative position error
||X_mixed - X_fp64|| / ||X_fp64|| at most 1e-5, and the per-particle
relative error |x_mixed - x_fp64| / |x_fp64| at most 1e-5 for 99% of the
particles.  The largest per-particle error is bounded at 1e-4: a particle
whose contact with the moving platen starts one step apart in the two modes
is displaced by about v dt = 5e-7 m.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_POS_GATE = 1e-5


def _min_image(d, sc):
    d = d.copy()
    L = (sc.domain_max[0] - sc.domain_min[0], sc.domain_max[1] - sc.domain_min[1])
    for k, on in enumerate((sc.periodic_x, sc.periodic_y)):
        if on:
            d[:, k] -= L[k] * np.round(d[:, k] / L[k])
    return d


def test_mixed_detection_matches_fp64(fundem):
    from fundem_b200 import workloads
    sim, sc, info = workloads.bonded_column(n=2048, footprint=(16, 16), seed=3)
    sim.close()
    out = {}
    for prec in (fundem.FP64, fundem.FP32_MIXED):
        s = fundem.Simulation.from_scenario(sc, precision=prec)
        s.detect()
        out[prec] = (s.contacts(fundem.PP), s.contacts(fundem.PW))
        s.close()
    for k in range(2):
        a, b = out[fundem.FP64][k], out[fundem.FP32_MIXED][k]
        ka = set(zip(a["master"].tolist(), a["slave"].tolist()))
        kb = set(zip(b["master"].tolist(), b["slave"].tolist()))
        # only nodes within single-precision rounding of the surface may differ
        for key in ka ^ kb:
            src = a if key in ka else b
            i = np.nonzero((src["master"] == key[0]) & (src["slave"] == key[1]))[0][0]
            assert abs(src["overlap"][i]) < 1e-9
        common = sorted(ka & kb)
        ia = {key: i for i, key in enumerate(zip(a["master"].tolist(), a["slave"].tolist()))}
        ib = {key: i for i, key in enumerate(zip(b["master"].tolist(), b["slave"].tolist()))}
        if common:
            oa = np.array([a["overlap"][ia[c]] for c in common])
            ob = np.array([b["overlap"][ib[c]] for c in common])
            assert np.abs(oa - ob).max() < 1e-9  # metres; nodes sit ~1e-3 m from the centre
            na = np.array([a["normal"][ia[c]] for c in common])
            nb = np.array([b["normal"][ib[c]] for c in common])
            assert np.abs(na - nb).max() < 1e-4


def test_mixed_position_error_after_1000_steps(fundem):
    from fundem_b200 import workloads
    sim, sc, info = workloads.bonded_column(n=16384, footprint=(32, 32), seed=1)
    sim.close()
    st = {}
    for prec in (fundem.FP64, fundem.FP32_MIXED):
        s = fundem.Simulation.from_scenario(sc, precision=prec, records=False)
        s.detect()
        s.step(1000)
        s.sync()
        st[prec] = s.state()
        assert s.num_contacts(fundem.PP) > 0
        s.close()
    a, b = st[fundem.FP64], st[fundem.FP32_MIXED]
    d = _min_image(a["pos"] - b["pos"], sc)
    dx = np.linalg.norm(d, axis=1)
    rel = dx / np.linalg.norm(a["pos"], axis=1)
    assert np.linalg.norm(d) / np.linalg.norm(a["pos"]) <= REL_POS_GATE
    assert np.percentile(rel, 99) <= REL_POS_GATE, np.percentile(rel, 99)
    assert rel.max() <= 10 * REL_POS_GATE, rel.max()


def test_mixed_forces_one_step(fundem):
    """From the same state, one step's forces agree with FP64 within 1e-4 of
    the largest force: the single-precision trilinear value carries an
    absolute error of about 5e-11 m (corner values of about the grid spacing,
    7e-5 m, rounded to 24 bits), which the normal stiffness turns into about
    1e-6 N per node contact, against forces of order 0.1 N."""
    from fundem_b200 import workloads
    sim, sc, info = workloads.bonded_column(n=16384, footprint=(32, 32), seed=1)
    sim.step(300)  # into the compression phase
    st0 = sim.state()
    sim.close()
    sc.particles.pos, sc.particles.vel, sc.particles.quat = st0["pos"], st0["vel"], st0["quat"]
    f = {}
    for prec in (fundem.FP64, fundem.FP32_MIXED):
        s = fundem.Simulation.from_scenario(sc, precision=prec, records=False)
        s.detect()
        s.step(1)
        s.sync()
        f[prec] = s.state()["force"]
        s.close()
    fa, fb = f[fundem.FP64], f[fundem.FP32_MIXED]
    assert np.abs(fa).max() > 0
    assert np.abs(fa - fb).max() <= 1e-4 * np.abs(fa).max()


def test_precision_switch_between_steps(fundem):
    from fundem_b200 import workloads
    sim, sc, info = workloads.bonded_column(n=2048, footprint=(16, 16), seed=5)
    sim.step(10)
    sim.set_precision(fundem.FP32_MIXED)
    sim.step(10)
    sim.set_precision(fundem.FP64)
    sim.step(10)
    sim.sync()
    st = sim.state()
    assert np.all(np.isfinite(st["pos"])) and np.all(np.isfinite(st["force"]))
    sim.close()
