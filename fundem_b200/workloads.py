"""Benchmark workloads.

`bonded_column` builds the scaled, periodic, bonded workload in the
reference's two-phase pattern (a settling solve followed by a second solve,
LSSolver.h:440-467 run twice as apps/tutorial/LSParticleRolling.cpp:154-171
does):

1. N superellipsoids from 8 templates (semi-axes uniform in [0.8, 1.2] mm,
   exponents in {2, 4}, 32^3 SDFs, 642 nodes) on a jittered lattice,
   periodic in x and y, over a floor wall, with the top platen parked above
   the bed.  Random orientations are re-drawn, and remaining overlapping
   pairs pushed apart, with the library's own detection until no overlap
   exceeds 2 um.
2. Settle: the library's own steps under gravity until the bed is at rest
   (kinetic energy below 1e-4 of its peak during the fall) -- a settled,
   contact-rich bed with several node contacts per particle.
3. The platen is placed 1 um above the highest surface node, V-model bonds
   (E = 1e8 Pa, tensile strength 1e6 Pa, length = centre distance) join every
   pair whose surface gap is below 0.05 of the mean diameter, and the platen
   starts down at 1 m/s with dt = 5e-7 s.

No public dataset is involved; the state is seeded.
"""
from __future__ import annotations

import numpy as np

from . import scenario as S


def _owner(node_base, nodes):
    return np.searchsorted(node_base, nodes, side="right") - 1


def _node_base(sc):
    counts = np.array([len(sc.particle_geometries[g].nodes) for g in sc.particles.geo], np.int64)
    nb = np.zeros(len(counts), np.int64)
    nb[1:] = np.cumsum(counts)[:-1]
    return nb


def resolve_on_gpu(sim, sc, rng, tol=0.0, redraw_rounds=40, max_rounds=400, log=None):
    """Reduce interpenetrations to at most `tol` with the library's own
    detection: first re-draw the orientation of one particle of every pair
    overlapping by more than `tol`, then push the remaining pairs apart along
    their contact normals.  Pairs pushed apart end with overlaps just under
    `tol`, which leaves a jammed packing with small contacts.  Returns
    (particles re-oriented, orientations, positions)."""
    nb = _node_base(sc)
    st = sim.state()
    quat = st["quat"].copy()
    pos = st["pos"].copy()
    moved = set()
    n = len(pos)
    for r in range(max_rounds):
        sim.detect()
        c = sim.contacts(0)
        deep = c["overlap"] > tol
        if not np.any(deep):
            if log:
                log(f"resolve: done after {r} rounds, {len(c['master'])} node contacts within {tol:g}")
            return len(moved), quat, pos
        c = {k: v[deep] for k, v in c.items()}
        a = _owner(nb, c["master"])
        b = c["slave"]
        if r < redraw_rounds:
            pick = np.unique(np.where(rng.random(len(a)) < 0.5, a, b))
            quat[pick] = S.random_quaternions(rng, len(pick))
            moved.update(pick.tolist())
            sim.set_state(quat=quat)
        else:
            # deepest overlap per pair, applied symmetrically along the normal
            # (the normal points out of b toward a's node)
            key = a.astype(np.int64) * n + b
            order = np.lexsort((-c["overlap"], key))
            ks = key[order]
            first = np.ones(len(order), bool)
            first[1:] = ks[1:] != ks[:-1]
            sel = order[first]
            push = (0.5 * (c["overlap"][sel] - 0.5 * tol) + 1e-8)[:, None] * c["normal"][sel]
            d = np.zeros_like(pos)
            np.add.at(d, a[sel], push)
            np.add.at(d, b[sel], -push)
            pos += d
            sim.set_state(pos=pos)
        if log and (r % 10 == 0):
            log(f"resolve round {r}: {len(c['master'])} node contacts")
    raise RuntimeError("packing did not resolve")


def _rotation_rows(q):
    """Rotation matrices (k, 3, 3) of scalar-first unit quaternions."""
    q0, q1, q2, q3 = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    R = np.empty((len(q), 3, 3))
    R[:, 0, 0] = 1 - 2 * (q2 * q2 + q3 * q3); R[:, 0, 1] = 2 * (q1 * q2 - q0 * q3); R[:, 0, 2] = 2 * (q1 * q3 + q0 * q2)
    R[:, 1, 0] = 2 * (q1 * q2 + q0 * q3); R[:, 1, 1] = 1 - 2 * (q1 * q1 + q3 * q3); R[:, 1, 2] = 2 * (q2 * q3 - q0 * q1)
    R[:, 2, 0] = 2 * (q1 * q3 - q0 * q2); R[:, 2, 1] = 2 * (q2 * q3 + q0 * q1); R[:, 2, 2] = 1 - 2 * (q1 * q1 + q2 * q2)
    return R


def top_of_bed(geos, geo, pos, quat):
    """World height of the highest surface node over all particles: bounding
    spheres select the particles that can hold it, their nodes are rotated
    exactly."""
    r = np.array([S.node_radius(g) for g in geos])[geo]
    zb = pos[:, 2] + r
    cand = np.nonzero(zb >= zb.max() - 2.0 * r.max())[0]
    best = -np.inf
    for g in np.unique(geo[cand]):
        idx = cand[geo[cand] == g]
        Rz = _rotation_rows(quat[idx])[:, 2, :]            # (k, 3): z row
        z = Rz @ np.asarray(geos[g].nodes, float).T         # (k, nodes)
        best = max(best, float(np.max(z.max(axis=1) + pos[idx, 2])))
    return best


def settle(sim, masses, dt, max_steps, chunk=500, ke_frac=1e-4, log=None):
    """Step under gravity (the library's own steps) until the kinetic energy
    falls below ke_frac of the largest value seen during the settle (the
    energy of the fall), checked every `chunk` steps, or max_steps.  Returns
    a record of the settle."""
    steps, hist = 0, []
    ke_peak, ke, vmax = 0.0, np.inf, np.inf
    while steps < max_steps:
        k = min(chunk, max_steps - steps)
        sim.step(k, dt=dt)
        steps += k
        v = sim.state()["vel"]
        speed = np.linalg.norm(v, axis=1)
        vmax = float(speed.max())
        ke = float(0.5 * np.sum(masses * speed ** 2))
        ke_peak = max(ke_peak, ke)
        nc = sim.num_contacts(0)
        hist.append((steps, ke, vmax, nc))
        if log:
            log(f"settle {steps} steps: kinetic energy {ke:.3e} J, peak speed {vmax:.3e} m/s, "
                f"{nc} particle node contacts")
        if steps >= 4 * chunk and ke < ke_frac * ke_peak:
            break
    return {"steps": steps, "dt": dt, "peak_speed": vmax, "kinetic_energy": ke, "kinetic_energy_peak": ke_peak,
            "settled": bool(ke < ke_frac * ke_peak), "history": hist}


def coordination(sim, sc, n):
    """Mean number of distinct particle partners in node contact per particle
    (particle-particle list; each touching pair counts for both particles)."""
    c = sim.contacts(0)
    if len(c["master"]) == 0:
        return 0.0
    a = _owner(_node_base(sc), c["master"])
    pairs = np.unique(np.minimum(a, c["slave"]).astype(np.int64) * n + np.maximum(a, c["slave"]))
    return 2.0 * len(pairs) / n


def bonded_column(n=262144, footprint=(128, 128), seed=1, pitch=2.42e-3, jitter=0.02e-3, n_templates=8,
                  dt=5e-7, young=1e8, poisson=0.3, tensile=1e6, gap_frac=0.05, bond_radius_frac=0.3,
                  platen_speed=1.0, overlap_tol=2e-6, settle_dt=5e-6, settle_steps=24000, settle_ke_frac=1e-4,
                  device=0, precision=0, records=False, log=None):
    """Build the workload and return (Simulation, Scenario, info).  The
    returned scenario holds the settled state (positions, orientations,
    velocities), the bonds and the moving platen; the simulation also keeps
    the contact history of the settle."""
    from . import Simulation
    rng = np.random.default_rng(seed)
    geos = S.superellipsoid_templates(rng, n_templates, n=32, level=3, density=2500.0, explicit_mass=True)
    nx, ny = footprint
    nz = int(np.ceil(n / (nx * ny)))
    box = np.array([nx, ny, nz]) * pitch
    pos = S.lattice_positions(rng, n, np.zeros(3), box + 1e-12, pitch, jitter)
    # lift the bed so no surface node starts below the floor
    rmax = max(S.node_radius(g) for g in geos)
    pos[:, 2] += rmax + 0.01 * pitch - 0.5 * pitch
    geo = rng.integers(0, n_templates, n).astype(np.int32)
    quat = S.random_quaternions(rng, n)
    objs = S.Objects(pos, np.zeros((n, 3)), np.zeros((n, 3)), quat, np.zeros(n, np.int32), geo)
    damping_ratio = 0.3
    e = float(np.exp(-np.pi * damping_ratio / np.sqrt(1 - damping_ratio ** 2)))
    # phase 1: the platen parked above the bed (centres of walls must lie
    # inside the domain: out-of-domain objects are no contact targets).
    # Without a settle (settle_steps = 0) the platen starts 1 um above the
    # highest node any lattice particle can reach and moves from the start.
    settling = settle_steps > 0
    motion = [(1, np.array([0.0, 0.0, -platen_speed]), np.zeros(3))]
    parked = float(np.max(pos[:, 2])) + rmax + (0.5e-3 if settling else 1e-6)
    ext = float(max(box[0], box[1])) * 1.05
    wall_geos = [S.plane_wall_template(ext), S.plane_wall_template(ext)]
    c = 0.5 * box
    walls = S.Objects(np.array([[c[0], c[1], 0.0], [c[0], c[1], parked]]), np.zeros((2, 3)), np.zeros((2, 3)),
                      np.array([S.WALL_QUAT["+z"], S.WALL_QUAT["-z"]]), np.zeros(2, np.int32),
                      np.array([0, 1], np.int32))
    sc = S.Scenario(domain_min=np.array([0.0, 0.0, -1e-3]), domain_max=np.array([box[0], box[1], parked + 1e-3]),
                    gravity=np.array([0.0, 0.0, -9.81]), dt=dt,
                    particle_materials=[(1e4, 0.8e4, 0.5, e)], wall_materials=[(0.5, e)],
                    particle_geometries=geos, wall_geometries=wall_geos, particles=objs, walls=walls,
                    wall_motion=[] if settling else motion, periodic_x=True, periodic_y=True, name="bonded_column")
    sim = Simulation.from_scenario(sc, device=device, precision=precision, records=True)
    moved, quat, pos = resolve_on_gpu(sim, sc, rng, tol=overlap_tol, log=log)
    sc.particles.quat = quat
    sc.particles.pos = pos
    rec = {"steps": 0, "peak_speed": None, "settled": False}
    coord, settled_contacts, top = None, None, parked
    if settling:
        # phase 2: settle under gravity
        sim.set_records(False)
        sim.detect()
        masses = np.array([g.mass for g in geos])[geo]
        rec = settle(sim, masses, settle_dt, settle_steps, ke_frac=settle_ke_frac, log=log)
        st = sim.state()
        sc.particles.pos, sc.particles.quat, sc.particles.vel = st["pos"], st["quat"], st["vel"]
        sc.particles.angvel = st["angvel"]
        coord = coordination(sim, sc, n)
        settled_contacts = sim.num_contacts(0)
        if log:
            log(f"settled: {settled_contacts} particle node contacts, coordination {coord:.2f}")
        # phase 3: platen 1 um above the highest surface node, moving down
        top = top_of_bed(geos, geo, st["pos"], st["quat"]) + 1e-6
        wst = sim.state(wall=True)
        sim.set_state(wall=True, pos=np.array([wst["pos"][0], [c[0], c[1], top]]))
        sim.set_wall_motion(1, motion[0][1], motion[0][2])
        sc.walls.pos = np.array([[c[0], c[1], 0.0], [c[0], c[1], top]])
        sc.wall_motion = motion
    # bonds between pairs whose surface gap is below gap_frac of the mean diameter
    d_mean = 2.0 * float(np.mean([np.mean(np.linalg.norm(g.nodes, axis=1)) for g in geos]))
    gap = gap_frac * d_mean
    sim.set_records(True)
    if log:
        log(f"platen at {top:.6f} m; bonding pairs with gaps below {gap:.3e} m")
    sim.detect_proximity(gap)
    if log:
        log(f"proximity detection: {sim.num_contacts(0)} node-partner pairs")
    cp = sim.contacts(0)
    nb = _node_base(sc)
    a = _owner(nb, cp["master"])
    b = cp["slave"]
    key = a.astype(np.int64) * n + b
    order = np.lexsort((-cp["overlap"], key))
    key_s = key[order]
    first = np.ones(len(order), bool)
    first[1:] = key_s[1:] != key_s[:-1]
    sel = order[first]
    nbond = len(sel)
    R = bond_radius_frac * 0.5 * d_mean
    # bond length: the distance between the two particle centres (the beam
    # joins the centres; a length of the order of the gap makes the bond's
    # shear stiffness, which scales as 1/L0^2, far stiffer than the contacts)
    L0 = np.linalg.norm(sc.particles.pos[a[sel]] - sc.particles.pos[b[sel]], axis=1)
    sim.add_bonds(a[sel], b[sel], cp["point"][sel], cp["normal"][sel], np.full(nbond, R), L0,
                  np.full(nbond, young), np.full(nbond, poisson), np.full(nbond, tensile), np.zeros(nbond),
                  np.zeros(nbond))
    sc.bonds = S.Bonds(a[sel].astype(np.int32), b[sel].astype(np.int32), cp["point"][sel], cp["normal"][sel],
                       np.full(nbond, R), L0, np.full(nbond, young), np.full(nbond, poisson),
                       np.full(nbond, tensile), np.zeros(nbond), np.zeros(nbond))
    # the proximity detection left gap partners in the history lists; the
    # settled contacts' springs are restored by detecting on the settled state
    if log:
        log(f"{nbond} bonds")
    sim.setup(sc.domain_min, sc.domain_max)
    sim.set_records(records)
    sim.detect()
    info = dict(n=n, templates=n_templates, resampled=moved, bonds=nbond, gap=gap, d_mean=d_mean,
                footprint=[nx, ny], layers=nz, pitch=pitch, settle_steps=rec["steps"], settle_dt=settle_dt,
                settle_peak_speed=rec["peak_speed"], settle_kinetic_energy=rec.get("kinetic_energy"),
                settle_kinetic_energy_peak=rec.get("kinetic_energy_peak"), settled=rec["settled"], coordination=coord,
                settled_node_contacts=settled_contacts, platen_top=top)
    return sim, sc, info


def adjoint_pour(n=4096, seed=0, n_templates=2, box=(40e-3, 40e-3, 80e-3), pitch=2.8e-3, dt=1e-6,
                 overlap_tol=2e-6, settle_steps=0, settle_dt=5e-6, settle_ke_frac=1e-3, device=0, log=None):
    """The adjoint workload: n superellipsoids (the small pour's distributions,
    2 templates, 32^3 SDFs, 642 nodes) on a jittered lattice in a box of six
    plane walls, dt = 1e-6 s, orientations re-drawn on the GPU until no
    overlap exceeds overlap_tol.  With settle_steps > 0 the lattice is then
    poured (the library's own steps under gravity at settle_dt, untimed)
    until its kinetic energy falls below settle_ke_frac of the fall's peak
    or settle_steps, and the scenario carries the settled state, so that a
    window started from it is full of particle and wall contacts.  Returns
    (Simulation, Scenario)."""
    from . import Simulation
    sc = S.pour(n=n, n_templates=n_templates, seed=seed, box=box, pitch=pitch, dt=dt, explicit_mass=True,
                resolve=False, name="adjoint_pour")
    rng = np.random.default_rng(seed + 1)
    sim = Simulation.from_scenario(sc, device=device, records=True)
    moved, quat, pos = resolve_on_gpu(sim, sc, rng, tol=overlap_tol, log=log)
    sc.particles.quat = quat
    sc.particles.pos = pos
    sim.set_state(quat=quat, pos=pos)
    sim.set_records(False)
    sim.detect()
    if settle_steps > 0:
        masses = np.array([g.mass for g in sc.particle_geometries])[sc.particles.geo]
        rec = settle(sim, masses, settle_dt, settle_steps, ke_frac=settle_ke_frac, log=log)
        st = sim.state()
        sc.particles.pos, sc.particles.vel = st["pos"].copy(), st["vel"].copy()
        sc.particles.angvel, sc.particles.quat = st["angvel"].copy(), st["quat"].copy()
        sc.settle = {k: rec[k] for k in ("steps", "dt", "settled", "kinetic_energy", "kinetic_energy_peak")}
    return sim, sc
