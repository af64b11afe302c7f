"""Scenario and dump files of the reference driver (oracle/ref_driver.cpp).

TEST INFRASTRUCTURE ONLY.  `write_reference_scenario` serialises a Scenario
for the driver; `read_dump` / `read_geometry` parse what the driver writes.
All values little-endian; see ref_driver.cpp for the reading side.
"""
from __future__ import annotations

import struct

import numpy as np

MAGIC = 0x43534446
VERSION = 1
KINDS = ("pp", "pw", "gx", "gy", "gxy")
# the sector images' lists follow the bonds in a dump, when the run has them
SECTOR_KINDS = ("gr90", "gr180", "gr270")


class _W:
    def __init__(self):
        self.parts = []

    def i32(self, *v):
        self.parts.append(struct.pack("<%di" % len(v), *[int(x) for x in v]))

    def u32(self, v):
        self.parts.append(struct.pack("<I", v))

    def i64(self, v):
        self.parts.append(struct.pack("<q", int(v)))

    def f64(self, *v):
        self.parts.append(struct.pack("<%dd" % len(v), *[float(x) for x in v]))

    def arr(self, a, dtype):
        self.parts.append(np.ascontiguousarray(a, dtype=dtype).tobytes())

    def bytes(self):
        return b"".join(self.parts)


def write_reference_scenario(sc, path, n_steps, dump_steps=()):
    w = _W()
    w.u32(MAGIC)
    w.u32(VERSION)
    w.f64(*sc.domain_min)
    w.f64(*sc.domain_max)
    w.f64(*sc.gravity)
    w.f64(sc.dt)
    w.i64(n_steps)
    # periodicity flags; bit 1 of the first one asks for sector periodicity
    # (kept inside the x flag so that scenario files without it are unchanged)
    w.i32(int(sc.periodic_x) | (2 if getattr(sc, "periodic_sector", False) else 0), int(sc.periodic_y))
    w.i32(len(dump_steps))
    for s in dump_steps:
        w.i32(s)
    w.i32(len(sc.particle_materials))
    for m in sc.particle_materials:
        w.f64(*m)
    w.i32(len(sc.wall_materials))
    for m in sc.wall_materials:
        w.f64(*m)

    def geo(g, particle):
        if particle:
            mode = 1 if g.density is not None else 0
            w.i32(mode)
            w.f64(g.mass)
            w.f64(*np.asarray(g.inertia, float).reshape(6))
            w.f64(g.density if g.density is not None else 0.0)
        w.f64(*np.asarray(g.origin, float))
        w.f64(g.spacing)
        w.i32(*np.asarray(g.size, int))
        w.arr(g.sdf, "<f8")
        w.i32(len(g.nodes))
        w.arr(g.nodes, "<f8")
        w.i32(len(g.tris))
        w.arr(g.tris, "<i4")

    for gi, g in enumerate(sc.particle_geometries):
        if g.density is not None:
            mats = np.unique(sc.particles.mat[sc.particles.geo == gi])
            if len(mats) > 1:
                raise ValueError("addParticleCluster gives one material to all particles of a geometry")
    w.i32(len(sc.particle_geometries))
    for g in sc.particle_geometries:
        geo(g, True)
    w.i32(len(sc.wall_geometries))
    for g in sc.wall_geometries:
        geo(g, False)

    def objs(o):
        w.i32(len(o))
        for i in range(len(o)):
            w.f64(*o.pos[i], *o.vel[i], *o.angvel[i], *o.quat[i])
            w.i32(o.mat[i], o.geo[i])

    objs(sc.particles)
    objs(sc.walls)
    w.i32(len(sc.wall_motion))
    for (idx, v, a) in sc.wall_motion:
        w.i32(idx)
        w.f64(*v, *a)
    B = sc.bonds
    w.i32(len(B))
    for k in range(len(B)):
        w.i32(B.master[k], B.slave[k])
        w.f64(*B.point[k], *B.normal[k], B.radius[k], B.length[k], B.young[k], B.poisson[k], B.tensile[k],
              B.cohesion[k], B.friction[k])
    with open(path, "wb") as f:
        f.write(w.bytes())


class _R:
    def __init__(self, data):
        self.b = data
        self.o = 0

    def get(self, fmt):
        v = struct.unpack_from("<" + fmt, self.b, self.o)
        self.o += struct.calcsize("<" + fmt)
        return v

    def arr(self, dtype, n, shape=None):
        dt = np.dtype(dtype)
        a = np.frombuffer(self.b, dtype=dt, count=n, offset=self.o).copy()
        self.o += dt.itemsize * n
        return a if shape is None else a.reshape(shape)


def read_dump(path):
    with open(path, "rb") as f:
        r = _R(f.read())
    step, = r.get("q")
    time, = r.get("d")
    nP, nW = r.get("ii")
    d = dict(step=step, time=time)
    d["pos"] = r.arr("<f8", 3 * nP, (nP, 3))
    d["vel"] = r.arr("<f8", 3 * nP, (nP, 3))
    d["angvel"] = r.arr("<f8", 3 * nP, (nP, 3))
    d["quat"] = r.arr("<f8", 4 * nP, (nP, 4))
    d["force"] = r.arr("<f8", 3 * nP, (nP, 3))
    d["torque"] = r.arr("<f8", 3 * nP, (nP, 3))
    d["wall_pos"] = r.arr("<f8", 3 * nW, (nW, 3))
    d["wall_quat"] = r.arr("<f8", 4 * nW, (nW, 4))

    def contacts():
        n, = r.get("q")
        return dict(master=r.arr("<i4", n), slave=r.arr("<i4", n), point=r.arr("<f8", 3 * n, (n, 3)),
                    normal=r.arr("<f8", 3 * n, (n, 3)), overlap=r.arr("<f8", n), spring=r.arr("<f8", 3 * n, (n, 3)),
                    en=r.arr("<f8", n), es=r.arr("<f8", n))

    for k in KINDS:
        d[k] = contacts()
    nb, = r.get("q")
    d["bonds"] = dict(activated=r.arr("<i4", nb), point=r.arr("<f8", 3 * nb, (nb, 3)), un=r.arr("<f8", nb),
                      us=r.arr("<f8", nb), ub=r.arr("<f8", nb), ut=r.arr("<f8", nb), sn=r.arr("<f8", nb),
                      ss=r.arr("<f8", nb))
    if r.o < len(r.b):
        for k in SECTOR_KINDS:
            d[k] = contacts()
    return d


def read_geometry(path):
    with open(path, "rb") as f:
        r = _R(f.read())
    n, = r.get("i")
    g = dict(radius=r.arr("<f8", n), inv_mass=r.arr("<f8", n), inertia=r.arr("<f8", 6 * n, (n, 6)),
             inv_inertia=r.arr("<f8", 6 * n, (n, 6)), origin=r.arr("<f8", 3 * n, (n, 3)))
    nn, = r.get("q")
    g["nodes"] = r.arr("<f8", 3 * nn, (nn, 3))
    nP, = r.get("i")
    g["pos"] = r.arr("<f8", 3 * nP, (nP, 3))
    g["grid_min"] = np.array(r.get("ddd"))
    g["grid_max"] = np.array(r.get("ddd"))
    g["grid_inv"] = np.array(r.get("ddd"))
    g["grid_size"] = np.array(r.get("iii"))
    return g
