"""Seeded scenarios used for parity (oracle vs CUDA path vs the reference's
own CUDA build).  Small enough for the CPU oracle to finish in seconds, and
arranged so every code path sees work:

* `cluster`: cm-scale superellipsoids (non-zero inverse inertia, so rotations
  are integrated) compressed into overlap inside a box of six plane walls,
  random linear and angular velocities, friction, one geometry registered
  through a density (mass properties from the SDF) and one particle whose
  centre sits above the domain (invisible as a contact target).
* `periodic`: a column periodic in x and y on a floor wall with a moving top
  platen and V-model bonds between near neighbours.
* `sector`: a quarter-sector pile periodic about the z axis through the
  domain's min corner (addPeriodicBoundarySector), cm-scale rotating bodies
  on a floor wall; one body starts just outside the x face, so the first
  step turns it back into the sector.
* `pour_mm`: mm-scale config-0 shapes (the inverse inertia falls under the
  1e-30 determinant threshold and is zero).
* `sphere`: the sphere-on-plane case of the reference's test app.
* `pour1000`: the small pour as configured (1,000 superellipsoids from 4
  templates, 32^3 grids, 642 nodes, six plane walls of a 20 x 20 x 40 mm box,
  seed 0), its lattice pulled 3% towards the box centre and given small
  random velocities, so that contacts start at once.
"""
from __future__ import annotations

import copy

import numpy as np

from fundem_b200 import scenario as S


def _compress(objs, centre, factor):
    objs.pos[:] = centre + (objs.pos - centre) * factor


def cluster(seed=3, n=48, grid_n=16, level=2):
    rng = np.random.default_rng(seed)
    geos = S.superellipsoid_templates(rng, 3, lo=8e-3, hi=12e-3, n=grid_n, level=level, density=2500.0,
                                      explicit_mass=True)
    # one template registered through its density
    g = S.superellipsoid_templates(rng, 1, lo=8e-3, hi=12e-3, n=grid_n, level=level, density=2000.0)[0]
    geos.append(g)
    pitch = 2 * max(S.node_radius(x) for x in geos) * 1.02
    side = int(np.ceil(n ** (1 / 3)))
    box = np.array([side, side, int(np.ceil(n / side / side))]) * pitch
    pos = S.lattice_positions(rng, n, np.zeros(3), box + 1e-9, pitch, 0.02 * pitch)
    geo = np.sort(rng.integers(0, 4, n)).astype(np.int32)
    quat = S.random_quaternions(rng, n)
    vel = rng.normal(0, 0.3, (n, 3))
    angvel = rng.normal(0, 20.0, (n, 3))
    objs = S.Objects(pos, vel, angvel, quat, np.zeros(n, np.int32), geo)
    f = 0.84
    _compress(objs, 0.5 * box, f)
    # walls just inside the outermost particles' extents
    reach = f * (np.array([side, side, int(np.ceil(n / side / side))]) - 1) / 2 * pitch + 0.42 * pitch
    lo, hi = 0.5 * box - reach, 0.5 * box + reach
    # open top (five walls); the domain ends just above the top layer's
    # centres and one particle is lifted so its centre leaves the domain
    wall_geos, walls = S.box_walls(lo, hi, faces=("+z", "+x", "-x", "+y", "-y"))
    dom_lo, dom_hi = lo - 0.3 * pitch, hi + 0.3 * pitch
    dom_hi[2] = objs.pos[:, 2].max() + 0.05 * pitch
    objs.pos[-1, 2] = dom_hi[2] + 0.1 * pitch
    sc = S.Scenario(domain_min=dom_lo, domain_max=dom_hi, gravity=np.array([0.0, 0.0, -9.81]), dt=2e-5,
                    particle_materials=[(2e4, 1.6e4, 0.5, 0.4), (3e4, 1e4, 0.3, 0.7)], wall_materials=[(0.4, 0.6)],
                    particle_geometries=geos, wall_geometries=wall_geos, particles=objs, walls=walls,
                    name="cluster")
    sc.particles.mat[::3] = 1
    # addParticleCluster takes one material for all of a geometry's particles
    sc.particles.mat[sc.particles.geo == 3] = 0
    return sc


def periodic(seed=5, nx=4, ny=4, nz=3, grid_n=16, level=2):
    rng = np.random.default_rng(seed)
    geos = S.superellipsoid_templates(rng, 2, lo=8e-3, hi=12e-3, n=grid_n, level=level, density=2500.0,
                                      explicit_mass=True)
    pitch = 2 * max(S.node_radius(x) for x in geos) * 0.70
    n = nx * ny * nz
    box = np.array([nx, ny, nz]) * pitch
    pos = S.lattice_positions(rng, n, np.zeros(3), box + 1e-9, pitch, 0.03 * pitch)
    pos[:, 2] += 0.2 * pitch
    geo = rng.integers(0, 2, n).astype(np.int32)
    objs = S.Objects(pos, rng.normal(0, 0.2, (n, 3)), rng.normal(0, 10.0, (n, 3)), S.random_quaternions(rng, n),
                     np.zeros(n, np.int32), geo)
    top = box[2] + 0.4 * pitch
    ext = float(max(box[0], box[1])) * 1.1
    wall_geos = [S.plane_wall_template(ext), S.plane_wall_template(ext)]
    c = 0.5 * box
    walls = S.Objects(np.array([[c[0], c[1], 0.15 * pitch], [c[0], c[1], top]]), np.zeros((2, 3)), np.zeros((2, 3)),
                      np.array([S.WALL_QUAT["+z"], S.WALL_QUAT["-z"]]), np.zeros(2, np.int32),
                      np.array([0, 1], np.int32))
    # bonds between bounding-sphere neighbours that do not cross the seam
    radius = np.array([S.node_radius(geos[g]) for g in geo])
    pairs = S.candidate_pairs(objs.pos, radius, margin=0.05 * pitch)
    d = objs.pos[pairs[:, 1]] - objs.pos[pairs[:, 0]]
    pairs = pairs[np.all(np.abs(d[:, :2]) < 0.5 * box[:2], axis=1)]
    sel = pairs[rng.random(len(pairs)) < 0.5]
    mid = 0.5 * (objs.pos[sel[:, 0]] + objs.pos[sel[:, 1]])
    nrm = objs.pos[sel[:, 0]] - objs.pos[sel[:, 1]]
    nb = len(sel)
    bonds = S.Bonds(sel[:, 0].astype(np.int32), sel[:, 1].astype(np.int32), mid, nrm, np.full(nb, 0.15 * pitch),
                    np.full(nb, 0.1 * pitch), np.full(nb, 2e6), np.full(nb, 0.3), np.full(nb, 2e4), np.zeros(nb),
                    np.zeros(nb))
    dom_lo = np.array([0.0, 0.0, -0.1 * pitch])
    dom_hi = np.array([box[0], box[1], top + 0.2 * pitch])
    return S.Scenario(domain_min=dom_lo, domain_max=dom_hi, gravity=np.array([0.0, 0.0, -9.81]), dt=2e-5,
                      particle_materials=[(2e4, 1.6e4, 0.5, 0.5)], wall_materials=[(0.5, 0.5)],
                      particle_geometries=geos, wall_geometries=wall_geos, particles=objs, walls=walls,
                      wall_motion=[(1, np.array([0.0, 0.0, -0.5]), np.zeros(3))], bonds=bonds,
                      periodic_x=True, periodic_y=True, name="periodic")


def sector(seed=11, nx=4, ny=4, nz=2, grid_n=16, level=2):
    rng = np.random.default_rng(seed)
    geos = S.superellipsoid_templates(rng, 2, lo=8e-3, hi=12e-3, n=grid_n, level=level, density=2500.0,
                                      explicit_mass=True)
    pitch = 2 * max(S.node_radius(x) for x in geos) * 0.72
    n = nx * ny * nz
    box = np.array([nx, ny, nz]) * pitch
    pos = S.lattice_positions(rng, n, np.zeros(3), box + 1e-9, pitch, 0.03 * pitch)
    pos[:, 2] += 0.2 * pitch
    # one body above the pile, just outside the x face
    pos[0] = [-0.05 * pitch, 1.5 * pitch, box[2] + 0.4 * pitch]
    # one body close to the axis, where it meets its own half-turned image
    pos[nx * ny, :2] = 0.3 * pitch
    geo = rng.integers(0, 2, n).astype(np.int32)
    objs = S.Objects(pos, rng.normal(0, 0.2, (n, 3)), rng.normal(0, 10.0, (n, 3)), S.random_quaternions(rng, n),
                     np.zeros(n, np.int32), geo)
    ext = float(max(box[0], box[1])) * 2.2
    wall_geos = [S.plane_wall_template(ext)]
    walls = S.Objects(np.array([[0.5 * box[0], 0.5 * box[1], 0.15 * pitch]]), np.zeros((1, 3)), np.zeros((1, 3)),
                      np.array([S.WALL_QUAT["+z"]]), np.zeros(1, np.int32), np.array([0], np.int32))
    dom_lo = np.array([0.0, 0.0, -0.1 * pitch])
    dom_hi = np.array([box[0], box[1], box[2] + 0.8 * pitch])
    return S.Scenario(domain_min=dom_lo, domain_max=dom_hi, gravity=np.array([0.0, 0.0, -9.81]), dt=2e-5,
                      particle_materials=[(2e4, 1.6e4, 0.5, 0.5)], wall_materials=[(0.5, 0.5)],
                      particle_geometries=geos, wall_geometries=wall_geos, particles=objs, walls=walls,
                      periodic_sector=True, name="sector")


def pour_mm(seed=0, n=64, grid_n=32, level=3):
    sc = S.pour(n=n, n_templates=4, seed=seed, box=(11e-3, 11e-3, 11e-3), pitch=2.7e-3, jitter=0.05e-3,
                init_speed=0.0, grid_n=grid_n, level=level, resolve=True, name="pour_mm")
    # pull the lattice together so surfaces interpenetrate a little
    _compress(sc.particles, np.array([5.5e-3, 5.5e-3, 5.5e-3]), 0.95)
    sc.particles.vel[:] = np.random.default_rng(seed).normal(0, 0.05, (n, 3))
    return sc


def sphere():
    return S.sphere_on_plane()


_POUR0 = {}


def pour_config0():
    """The small pour exactly as configured (scenario.pour() defaults).  Its
    host-side overlap resolution takes tens of seconds, so it is built once
    per process; each call returns an independent copy."""
    if "sc" not in _POUR0:
        _POUR0["sc"] = S.pour()
    return copy.deepcopy(_POUR0["sc"])


def pour1000(seed=0):
    sc = pour_config0()
    sc.name = "pour1000"
    _compress(sc.particles, np.array([10e-3, 10e-3, 20e-3]), 0.97)
    sc.particles.vel[:] = np.random.default_rng(seed).normal(0, 0.02, (len(sc.particles), 3))
    return sc


CASES = {"cluster": cluster, "periodic": periodic, "pour_mm": pour_mm, "sphere": sphere, "sector": sector,
         "pour1000": pour1000}
# in-loop steps the reference runs per case and the steps it dumps
REF_STEPS = {"cluster": (40, [1, 2, 3, 10, 11, 39, 40]), "periodic": (40, [1, 2, 3, 10, 11, 39, 40]),
             "sector": (40, [1, 2, 3, 10, 11, 39, 40]),
             "pour_mm": (20, [1, 2, 3, 19, 20]), "pour1000": (20, [1, 2, 10, 11, 19, 20]), "sphere": (10000, [1, 2, 4500, 4550, 4600, 4650, 4700, 9000, 10000])}
