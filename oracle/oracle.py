"""ctypes front end of the CPU oracle (oracle/fundem_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py, never by the product package.

`OracleWorld.from_scenario` loads a Scenario the way the reference's public
API would receive it: materials (LSSolver.h:33-42, 175-183), geometries with
explicit mass (LSSolver.h:58-76) or from a density through addParticleCluster
(LSSolver.h:125-165), particles, walls, wall motion (LSSolver.h:244-270),
bonds (LSSolver.h:296-317) and periodicity (LSSolver.h:384-414).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libfundem_oracle.so")

PP, PW, GX, GY, GXY = 0, 1, 2, 3, 4
GR90, GR180, GR270 = 5, 6, 7

_lib = None


def build():
    """Compile the oracle library (gcc, OpenMP, no FP contraction)."""
    os.makedirs(os.path.join(HERE, "_lib"), exist_ok=True)
    subprocess.check_call(["make", "-s", "-C", HERE, "oracle"])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        D = C.POINTER(C.c_double)
        I = C.POINTER(C.c_int)
        L.orc_create.restype = P
        L.orc_destroy.argtypes = [P]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_set_fma_mode.argtypes = [C.c_int]
        L.orc_set_fma_pattern.argtypes = [C.c_int]
        L.orc_add_material.argtypes = [P, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double]
        L.orc_add_geometry.argtypes = [P, C.c_int, C.c_double, D, D, C.c_double, I, D, C.c_int, D]
        L.orc_mass_properties.argtypes = [C.c_double, D, C.c_double, I, D, D, D, D]
        L.orc_inverse_sym.argtypes = [D, D]
        L.orc_add_object.argtypes = [P, C.c_int, D, D, D, D, C.c_int, C.c_int]
        L.orc_add_bond.argtypes = [P, C.c_int, C.c_int, D, D, C.c_double, C.c_double, C.c_double,
                                   C.c_double, C.c_double, C.c_double, C.c_double]
        L.orc_set_periodic.argtypes = [P, C.c_int, C.c_int]
        L.orc_set_sector.argtypes = [P, C.c_int]
        L.orc_set_inertia_mode.argtypes = [P, C.c_int]
        L.orc_set_damping_sqrt64.argtypes = [C.c_int]
        L.orc_setup.argtypes = [P, D, D]
        L.orc_initial_detect.argtypes = [P]
        L.orc_step.argtypes = [P, D, C.c_double]
        L.orc_half_kick.argtypes = [P, D, C.c_double]
        L.orc_front.argtypes = [P, D, C.c_double]
        L.orc_detect_and_force.argtypes = [P, C.c_double]
        L.orc_num_objects.argtypes = [P, C.c_int]
        L.orc_get_state.argtypes = [P, C.c_int, D, D, D, D, D, D]
        L.orc_set_state.argtypes = [P, C.c_int, D, D, D, D, D, D]
        L.orc_num_nodes.argtypes = [P]
        L.orc_num_nodes.restype = C.c_longlong
        L.orc_get_geometry.argtypes = [P, C.c_int, C.c_int, D, D, D, D]
        L.orc_get_grid.argtypes = [P, C.c_int, D, D, D, I]
        L.orc_num_contacts.argtypes = [P, C.c_int]
        L.orc_num_contacts.restype = C.c_longlong
        L.orc_get_contacts.argtypes = [P, C.c_int, I, I, D, D, D, D, D, D]
        L.orc_set_contacts.argtypes = [P, C.c_int, C.c_longlong, I, I, D]
        L.orc_num_bonds.argtypes = [P]
        L.orc_get_bonds.argtypes = [P, I, D, D, D, D, D, D, D]
        L.orc_set_bond_activation.argtypes = [P, I]
        L.orc_get_bond_params.argtypes = [P, D, D]
        _lib = L
    return _lib


def _d(a):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _i(a):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(C.c_int))


def _arr(x, n, dtype=np.float64):
    a = np.ascontiguousarray(np.asarray(x, dtype=dtype).reshape(-1))
    assert a.size == n, (a.size, n)
    return a


def mass_properties(density, origin, spacing, size, sdf):
    L = lib()
    m = np.zeros(1)
    c = np.zeros(3)
    I = np.zeros(6)
    L.orc_mass_properties(float(density), _d(_arr(origin, 3)), float(spacing), _i(_arr(size, 3, np.int32)),
                          _d(np.ascontiguousarray(sdf, dtype=np.float64)), _d(m), _d(c), _d(I))
    return float(m[0]), c, I


def inverse_sym(I6):
    out = np.zeros(6)
    lib().orc_inverse_sym(_d(_arr(I6, 6)), _d(out))
    return out


def set_threads(n):
    lib().orc_set_threads(int(n))


def set_fma_mode(m):
    lib().orc_set_fma_mode(int(m))


def set_fma_pattern(p):
    lib().orc_set_fma_pattern(int(p))


def _rot(q, v):
    qv = np.asarray(q[1:], float)
    t = 2.0 * np.cross(qv, v)
    return v + t * q[0] + np.cross(qv, t)


def prepared_particles(sc):
    """Apply addParticleCluster's centroid handling (LSSolver.h:145-164,
    LSSolver.h:567-585) to a scenario: per-geometry mass properties from the
    density, re-centred nodes and SDF origin, and particle positions offset
    by the (unnormalised) orientation applied to the centroid.  Returns
    (geometries as dicts, positions)."""
    geos = []
    pos = np.array(sc.particles.pos, dtype=np.float64, copy=True)
    for gi, g in enumerate(sc.particle_geometries):
        if g.density is None:
            geos.append(dict(mass=g.mass, inertia=np.asarray(g.inertia, float), origin=np.asarray(g.origin, float),
                             spacing=g.spacing, size=np.asarray(g.size, np.int32), sdf=g.sdf, nodes=g.nodes))
            continue
        m, c, I = mass_properties(g.density, g.origin, g.spacing, g.size, g.sdf)
        nodes = np.asarray(g.nodes, float) - c
        geos.append(dict(mass=m, inertia=I, origin=np.asarray(g.origin, float) - c, spacing=g.spacing,
                         size=np.asarray(g.size, np.int32), sdf=g.sdf, nodes=nodes))
        sel = np.nonzero(sc.particles.geo == gi)[0]
        for i in sel:
            pos[i] = pos[i] + _rot(sc.particles.quat[i], c)
    return geos, pos


class OracleWorld:
    def __init__(self):
        self.L = lib()
        self.w = self.L.orc_create()

    def close(self):
        if self.w:
            self.L.orc_destroy(self.w)
            self.w = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @classmethod
    def from_scenario(cls, sc, setup=True):
        o = cls()
        L, w = o.L, o.w
        for (kn, ks, mu, e) in sc.particle_materials:
            L.orc_add_material(w, 0, kn, ks, mu, e)
        for (mu, e) in sc.wall_materials:
            L.orc_add_material(w, 1, 0.0, 0.0, mu, e)
        geos, pos = prepared_particles(sc)
        for g in geos:
            nodes = np.ascontiguousarray(g["nodes"], dtype=np.float64)
            r = L.orc_add_geometry(w, 0, float(g["mass"]), _d(_arr(g["inertia"], 6)), _d(_arr(g["origin"], 3)),
                                   float(g["spacing"]), _i(_arr(g["size"], 3, np.int32)),
                                   _d(np.ascontiguousarray(g["sdf"], dtype=np.float64)), len(nodes), _d(nodes))
            assert r >= 0
        for g in sc.wall_geometries:
            nodes = np.ascontiguousarray(g.nodes, dtype=np.float64)
            r = L.orc_add_geometry(w, 1, 0.0, None, _d(_arr(g.origin, 3)), float(g.spacing),
                                   _i(_arr(g.size, 3, np.int32)), _d(np.ascontiguousarray(g.sdf, dtype=np.float64)),
                                   len(nodes), _d(nodes))
            assert r >= 0
        P = sc.particles
        for i in range(len(P)):
            r = L.orc_add_object(w, 0, _d(_arr(pos[i], 3)), _d(_arr(P.vel[i], 3)), _d(_arr(P.angvel[i], 3)),
                                 _d(_arr(P.quat[i], 4)), int(P.mat[i]), int(P.geo[i]))
            assert r >= 0
        W = sc.walls
        vel = np.array(W.vel, float, copy=True)
        ang = np.array(W.angvel, float, copy=True)
        for (idx, v, a) in sc.wall_motion:
            vel[idx] = v
            ang[idx] = a
        for i in range(len(W)):
            r = L.orc_add_object(w, 1, _d(_arr(W.pos[i], 3)), _d(_arr(vel[i], 3)), _d(_arr(ang[i], 3)),
                                 _d(_arr(W.quat[i], 4)), int(W.mat[i]), int(W.geo[i]))
            assert r >= 0
        B = sc.bonds
        for k in range(len(B)):
            L.orc_add_bond(w, int(B.master[k]), int(B.slave[k]), _d(_arr(B.point[k], 3)), _d(_arr(B.normal[k], 3)),
                           float(B.radius[k]), float(B.length[k]), float(B.young[k]), float(B.poisson[k]),
                           float(B.tensile[k]), float(B.cohesion[k]), float(B.friction[k]))
        L.orc_set_periodic(w, int(sc.periodic_x), int(sc.periodic_y))
        L.orc_set_sector(w, int(getattr(sc, "periodic_sector", False)))
        L.orc_set_inertia_mode(w, int(getattr(sc, "inertia", "reference") == "physical"))
        o.gravity = np.asarray(sc.gravity, float)
        o.dt = float(sc.dt)
        if setup:
            o.setup(sc.domain_min, sc.domain_max)
        return o

    # --- driving -------------------------------------------------------------
    def setup(self, minb, maxb):
        r = self.L.orc_setup(self.w, _d(_arr(minb, 3)), _d(_arr(maxb, 3)))
        assert r == 0

    def initial_detect(self):
        self.L.orc_initial_detect(self.w)

    def step(self, n=1, dt=None, gravity=None):
        dt = self.dt if dt is None else dt
        g = _arr(self.gravity if gravity is None else gravity, 3)
        for _ in range(n):
            self.L.orc_step(self.w, _d(g), float(dt))

    def half_kick(self, dt=None):
        self.L.orc_half_kick(self.w, _d(_arr(self.gravity, 3)), float(self.dt if dt is None else dt))

    def front(self, dt=None):
        self.L.orc_front(self.w, _d(_arr(self.gravity, 3)), float(self.dt if dt is None else dt))

    def detect_and_force(self, dt=None):
        self.L.orc_detect_and_force(self.w, float(self.dt if dt is None else dt))

    # --- state ---------------------------------------------------------------
    def num(self, wall=False):
        return self.L.orc_num_objects(self.w, int(wall))

    def num_nodes(self):
        return self.L.orc_num_nodes(self.w)

    def state(self, wall=False):
        n = self.num(wall)
        out = {k: np.zeros((n, 3)) for k in ("pos", "vel", "angvel", "force", "torque")}
        out["quat"] = np.zeros((n, 4))
        self.L.orc_get_state(self.w, int(wall), _d(out["pos"]), _d(out["vel"]), _d(out["angvel"]), _d(out["quat"]),
                             _d(out["force"]), _d(out["torque"]))
        return out

    def set_state(self, wall=False, pos=None, vel=None, angvel=None, quat=None, force=None, torque=None):
        n = self.num(wall)
        f = lambda a, k: None if a is None else _arr(a, n * k)
        self.L.orc_set_state(self.w, int(wall), _d(f(pos, 3)), _d(f(vel, 3)), _d(f(angvel, 3)), _d(f(quat, 4)),
                             _d(f(force, 3)), _d(f(torque, 3)))

    def geometry(self, geo, wall=False):
        r, im = np.zeros(1), np.zeros(1)
        I, Ii = np.zeros(6), np.zeros(6)
        self.L.orc_get_geometry(self.w, int(wall), int(geo), _d(r), _d(im), _d(I), _d(Ii))
        return dict(radius=float(r[0]), inv_mass=float(im[0]), inertia=I, inv_inertia=Ii)

    def grid(self, wall=False):
        mn, mx, inv = np.zeros(3), np.zeros(3), np.zeros(3)
        sz = np.zeros(3, np.int32)
        self.L.orc_get_grid(self.w, int(wall), _d(mn), _d(mx), _d(inv), _i(sz))
        return dict(min=mn, max=mx, inv_cell=inv, size=sz)

    def contacts(self, kind=PP):
        n = self.L.orc_num_contacts(self.w, kind)
        n = max(n, 0)
        c = dict(master=np.zeros(n, np.int32), slave=np.zeros(n, np.int32), point=np.zeros((n, 3)),
                 normal=np.zeros((n, 3)), overlap=np.zeros(n), spring=np.zeros((n, 3)), en=np.zeros(n),
                 es=np.zeros(n))
        if n:
            self.L.orc_get_contacts(self.w, kind, _i(c["master"]), _i(c["slave"]), _d(c["point"]), _d(c["normal"]),
                                    _d(c["overlap"]), _d(c["spring"]), _d(c["en"]), _d(c["es"]))
        return c

    def set_contacts(self, kind, master, slave, spring):
        master = np.ascontiguousarray(master, np.int32)
        slave = np.ascontiguousarray(slave, np.int32)
        spring = np.ascontiguousarray(spring, np.float64).reshape(-1)
        order = np.lexsort((np.arange(len(master)), master))
        master, slave = master[order], slave[order]
        spring = spring.reshape(-1, 3)[order].reshape(-1).copy()
        r = self.L.orc_set_contacts(self.w, kind, len(master), _i(master), _i(slave), _d(spring))
        assert r == 0

    def bonds(self):
        n = self.L.orc_num_bonds(self.w)
        b = dict(activated=np.zeros(n, np.int32), point=np.zeros((n, 3)), un=np.zeros(n), us=np.zeros(n),
                 ub=np.zeros(n), ut=np.zeros(n), sn=np.zeros(n), ss=np.zeros(n))
        if n:
            self.L.orc_get_bonds(self.w, _i(b["activated"]), _d(b["point"]), _d(b["un"]), _d(b["us"]), _d(b["ub"]),
                                 _d(b["ut"]), _d(b["sn"]), _d(b["ss"]))
        return b

    def set_bond_activation(self, act):
        self.L.orc_set_bond_activation(self.w, _i(np.ascontiguousarray(act, np.int32)))

    def bond_params(self):
        n = self.L.orc_num_bonds(self.w)
        b = np.zeros((n, 4))
        f = np.zeros((n, 8, 3))
        if n:
            self.L.orc_get_bond_params(self.w, _d(b), _d(f))
        return b, f
