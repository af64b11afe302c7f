"""The synthetic workloads against the configurations they stand in for
(no GPU: the scenarios are built on the host, before any resolve or bonding
step that needs the device).

* small pour: 1,000 superellipsoids from 4 templates (semi-axes in
  [0.8, 1.2] mm, exponents 2 or 4, 32^3 grids with spacing 1/14 of the
  largest semi-axis, 642 nodes), a jittered lattice in a 20 x 20 x 40 mm box
  of six walls, zero velocity, unit quaternions, kn = 1e4, kt = 0.8 kn,
  damping ratio 0.3, friction 0.5, density 2500, dt = 1e-6 s, gravity 9.81;
* calibration sweep: 256 pours with particle counts log-uniform in
  [500, 20,000], kn log-uniform in [5e3, 5e4], friction uniform in
  [0.2, 0.8], damping ratio uniform in [0.1, 0.5], fill ratio 0.4 or less.
"""
import numpy as np

from fundem_b200 import scenario as S


def _zeta(e):
    lr = np.log(e)
    return -lr / np.sqrt(lr * lr + np.pi * np.pi)


def test_small_pour():
    sc = S.pour(resolve=False)
    P = sc.particles
    assert len(P) == 1000
    assert len(sc.particle_geometries) == 4 and set(np.unique(P.geo)) <= {0, 1, 2, 3}
    for g in sc.particle_geometries:
        assert tuple(g.size) == (32, 32, 32)
        assert len(g.nodes) == 642
        extent = np.abs(g.nodes).max(axis=0)           # the surface nodes reach the semi-axes
        assert extent.max() <= 1.2e-3 * (1 + 1e-12) and extent.min() >= 0.8e-3 * 0.9
        assert abs(g.spacing * 14 - extent.max()) <= 0.02 * extent.max()
        assert g.density == 2500.0
    assert len(sc.walls) == 6
    lo, hi = P.pos.min(axis=0), P.pos.max(axis=0)
    assert np.all(lo > 0) and np.all(hi < [20e-3, 20e-3, 40e-3])
    assert not np.any(P.vel) and not np.any(P.angvel)
    assert np.allclose(np.linalg.norm(P.quat, axis=1), 1.0)
    (kn, ks, mu, e), = sc.particle_materials
    assert (kn, ks, mu) == (1e4, 0.8e4, 0.5)
    assert abs(_zeta(e) - 0.3) < 1e-12
    assert sc.dt == 1e-6 and np.array_equal(sc.gravity, [0.0, 0.0, -9.81])


def test_calibration_sweep():
    from fundem_b200 import batch
    scs, params = batch.calibration_scenarios()
    assert len(scs) == 256
    n = np.array([p["n"] for p in params])
    kn = np.array([p["kn"] for p in params])
    mu = np.array([p["mu"] for p in params])
    z = np.array([p["damping_ratio"] for p in params])
    assert n.min() >= 500 and n.max() <= 20000
    assert kn.min() >= 5e3 and kn.max() <= 5e4
    assert mu.min() >= 0.2 and mu.max() <= 0.8 and z.min() >= 0.1 and z.max() <= 0.5
    # log-uniform: the logarithms spread evenly over their range
    for x, a, b in ((n, 500, 20000), (kn, 5e3, 5e4)):
        u = (np.log(x) - np.log(a)) / (np.log(b) - np.log(a))
        assert abs(u.mean() - 0.5) < 0.06 and abs(np.median(u) - 0.5) < 0.1
    assert max(p["fill"] for p in params) <= 0.4 + 1e-12
    for sc, p in zip(scs, params):
        assert len(sc.particles) == p["n"] and len(sc.walls) == 6
        (k, ks, m, e), = sc.particle_materials
        assert k == p["kn"] and ks == 0.8 * k and m == p["mu"]
        assert abs(_zeta(e) - p["damping_ratio"]) < 1e-12


def test_bonded_column_parameters():
    """The benchmark's bonded periodic column (built on the device, so only
    its parameters are checked here): 262,144 particles from 8 templates,
    dt = 5e-7 s, bond modulus 1e8 Pa, tensile strength 1e6 Pa, bonds where
    the surface gap is below 0.05 of the mean diameter, a 1 m/s platen."""
    import inspect
    from fundem_b200 import workloads
    d = {k: v.default for k, v in inspect.signature(workloads.bonded_column).parameters.items()}
    assert d["n"] == 262144 and d["n_templates"] == 8 and d["dt"] == 5e-7
    assert d["young"] == 1e8 and d["tensile"] == 1e6 and d["gap_frac"] == 0.05 and d["platen_speed"] == 1.0
    a = {k: v.default for k, v in inspect.signature(workloads.adjoint_pour).parameters.items()}
    assert a["n"] == 4096 and a["n_templates"] == 2 and a["dt"] == 1e-6
