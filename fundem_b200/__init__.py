"""fundem_b200 -- B200-native level-set DEM timestep.

Python bindings over the C ABI of libfundem_b200.so (include/fundem_b200.h).
The library is built in-tree (`python -m fundem_b200.build`) and loaded from
fundem_b200/_lib/; there is no fallback: if the library or a CUDA device is
missing, the calls raise.
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libfundem_b200.so")

FP64, FP32_MIXED = 0, 1
INERTIA_REFERENCE, INERTIA_PHYSICAL = 0, 1
PP, PW, GX, GY, GXY = 0, 1, 2, 3, 4
GR90, GR180, GR270 = 5, 6, 7  # sector images

# every symbol declared in include/fundem_b200.h
EXPORTS = [
    "fundem_version", "fundem_status_string", "fundem_create", "fundem_destroy", "fundem_set_precision",
    "fundem_set_records", "fundem_add_material", "fundem_add_geometry", "fundem_mass_properties",
    "fundem_add_objects", "fundem_set_wall_motion", "fundem_move", "fundem_add_bonds", "fundem_set_periodic",
    "fundem_setup", "fundem_detect", "fundem_detect_proximity", "fundem_step", "fundem_step_begin", "fundem_step_end", "fundem_sync",
    "fundem_status_word", "fundem_num_objects", "fundem_get_objects", "fundem_set_objects",
    "fundem_device_view_get", "fundem_num_contacts", "fundem_get_contacts", "fundem_set_contacts",
    "fundem_num_pairs", "fundem_num_bonds", "fundem_get_bonds", "fundem_set_bond_activation",
    "fundem_get_geometry", "fundem_get_grid", "fundem_launch_count", "fundem_set_profiling",
    "fundem_kernel_time", "fundem_work_counters", "fundem_slot_counters", "fundem_set_launch_shape",
    "fundem_get_launch_shape", "fundem_prefix_sum", "fundem_prefix_sum_noalloc", "fundem_last_error",
    "fundem_adjoint_begin", "fundem_adjoint_forward", "fundem_adjoint_backward", "fundem_adjoint_end",
    "fundem_step_graph", "fundem_set_neighbour_list", "fundem_checkpoint_write", "fundem_checkpoint_read",
    "fundem_levelset_grid", "fundem_set_periodic_sector", "fundem_set_inertia_mode",
    "fundem_set_pair_cache", "fundem_pair_cache_stats", "fundem_set_wall_groups", "fundem_hash_sort",
    "fundem_adjoint_backward_rot", "fundem_contact_view_get", "fundem_bond_view_get",
]
TIMERS = {"integrate": 0, "hash": 1, "broad": 2, "narrow_pp": 3, "narrow_pw": 4, "ghost": 5, "reduce": 6}


class FundemError(RuntimeError):
    pass


class Shape(C.Structure):
    """fundem_shape: a shape whose signed-distance grid the GPU evaluates."""
    _fields_ = [("kind", C.c_int), ("positive_inside", C.c_int), ("param", C.c_double * 8),
                ("n_vertices", C.c_int), ("vertices", C.POINTER(C.c_double)),
                ("n_triangles", C.c_int), ("triangles", C.POINTER(C.c_int))]


SHAPES = {"superellipsoid": 0, "sphere": 1, "box": 2, "cylinder": 3, "mesh": 4}


class DeviceView(C.Structure):
    _fields_ = [("pos", C.c_void_p), ("vel", C.c_void_p), ("angvel", C.c_void_p), ("force", C.c_void_p),
                ("torque", C.c_void_p), ("quat", C.c_void_p), ("mat", C.c_void_p), ("geo", C.c_void_p),
                ("n", C.c_int)]


_lib = None


def lib():
    """Load libfundem_b200.so (raises when it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FundemError(f"{LIB_PATH} is missing: build it with `python -m fundem_b200.build`")
        L = C.CDLL(LIB_PATH)
        P, I, D, LL = C.c_void_p, C.c_int, C.POINTER(C.c_double), C.c_longlong
        IP = C.POINTER(C.c_int)
        L.fundem_version.restype = C.c_char_p
        L.fundem_status_string.restype = C.c_char_p
        L.fundem_status_string.argtypes = [I]
        L.fundem_create.argtypes = [C.POINTER(P), I, P]
        L.fundem_destroy.argtypes = [P]
        L.fundem_set_precision.argtypes = [P, I]
        L.fundem_set_records.argtypes = [P, I]
        L.fundem_add_material.argtypes = [P, I, C.c_double, C.c_double, C.c_double, C.c_double, IP]
        L.fundem_add_geometry.argtypes = [P, I, C.c_double, D, D, C.c_double, IP, D, I, D, IP]
        L.fundem_mass_properties.argtypes = [C.c_double, D, C.c_double, IP, D, D, D, D]
        L.fundem_add_objects.argtypes = [P, I, I, D, D, D, D, IP, IP]
        L.fundem_set_wall_motion.argtypes = [P, I, D, D]
        L.fundem_move.argtypes = [P, I, I, D]
        L.fundem_add_bonds.argtypes = [P, I, IP, IP, D, D, D, D, D, D, D, D, D]
        L.fundem_set_periodic.argtypes = [P, I, I]
        L.fundem_setup.argtypes = [P, D, D]
        L.fundem_detect.argtypes = [P]
        L.fundem_detect_proximity.argtypes = [P, C.c_double]
        L.fundem_step.argtypes = [P, I, D, C.c_double]
        L.fundem_step_begin.argtypes = [P, D, C.c_double]
        L.fundem_step_end.argtypes = [P, D, C.c_double]
        L.fundem_sync.argtypes = [P]
        L.fundem_status_word.argtypes = [P, C.POINTER(C.c_uint)]
        L.fundem_num_objects.argtypes = [P, I, IP]
        L.fundem_get_objects.argtypes = [P, I, D, D, D, D, D, D]
        L.fundem_set_objects.argtypes = [P, I, D, D, D, D, D, D]
        L.fundem_device_view_get.argtypes = [P, I, C.POINTER(DeviceView)]
        L.fundem_num_contacts.argtypes = [P, I, C.POINTER(LL)]
        L.fundem_get_contacts.argtypes = [P, I, IP, IP, D, D, D, D, D, D]
        L.fundem_set_contacts.argtypes = [P, I, LL, IP, IP, D]
        L.fundem_num_pairs.argtypes = [P, I, C.POINTER(LL)]
        L.fundem_num_bonds.argtypes = [P, IP]
        L.fundem_get_bonds.argtypes = [P, IP, D, D]
        L.fundem_set_bond_activation.argtypes = [P, IP]
        L.fundem_get_geometry.argtypes = [P, I, I, D, D, D, D]
        L.fundem_get_grid.argtypes = [P, I, D, D, D, IP]
        L.fundem_launch_count.argtypes = [P, C.POINTER(LL)]
        L.fundem_set_profiling.argtypes = [P, I]
        L.fundem_kernel_time.argtypes = [P, I, C.POINTER(C.c_double), C.POINTER(LL)]
        L.fundem_work_counters.argtypes = [P, C.POINTER(C.c_ulonglong)]
        L.fundem_slot_counters.argtypes = [P, C.POINTER(C.c_ulonglong)]
        L.fundem_set_launch_shape.argtypes = [P, C.POINTER(C.c_int)]
        L.fundem_get_launch_shape.argtypes = [P, C.POINTER(C.c_int)]
        L.fundem_prefix_sum.argtypes = [P, P, LL, P]
        L.fundem_prefix_sum_noalloc.argtypes = [P, P, LL, P]
        L.fundem_last_error.restype = C.c_char_p
        L.fundem_last_error.argtypes = [P]
        L.fundem_adjoint_begin.argtypes = [P, I]
        L.fundem_adjoint_forward.argtypes = [P, I, D, C.c_double]
        L.fundem_adjoint_backward.argtypes = [P, D, D, D, D]
        L.fundem_adjoint_backward_rot.argtypes = [P, D, D, D, D, D, D, D]
        L.fundem_adjoint_end.argtypes = [P]
        L.fundem_step_graph.argtypes = [P, I, D, C.c_double]
        L.fundem_set_neighbour_list.argtypes = [P, I]
        L.fundem_checkpoint_write.argtypes = [P, C.c_char_p]
        L.fundem_checkpoint_read.argtypes = [P, C.c_char_p]
        L.fundem_levelset_grid.argtypes = [I, P, C.POINTER(Shape), D, C.c_double, IP, D]
        L.fundem_set_periodic_sector.argtypes = [P, I]
        L.fundem_set_inertia_mode.argtypes = [P, I]
        L.fundem_set_pair_cache.argtypes = [P, I, C.c_double]
        L.fundem_set_wall_groups.argtypes = [P, I, IP, IP]
        L.fundem_hash_sort.argtypes = [P, I, LL, P, P, P]
        L.fundem_pair_cache_stats.argtypes = [P, C.POINTER(LL), C.POINTER(LL), C.POINTER(C.c_double)]
        _lib = L
    return _lib


def _d(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def _i(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_int))


def _f64(x, n=None):
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(-1))
    if n is not None:
        assert a.size == n, (a.size, n)
    return a


def _i32(x):
    return np.ascontiguousarray(np.asarray(x, dtype=np.int32).reshape(-1))


def _check(r, what=""):
    if r != 0:
        msg = lib().fundem_status_string(r).decode()
        raise FundemError(f"{what}: {msg} ({r})")


def mass_properties(density, origin, spacing, size, sdf):
    """Mass, centroid and inertia of a template from its SDF and a density
    (LSSolver.h:470-586), computed by the library's host code."""
    m, c, I = np.zeros(1), np.zeros(3), np.zeros(6)
    _check(lib().fundem_mass_properties(float(density), _d(_f64(origin, 3)), float(spacing), _i(_i32(size)),
                                        _d(_f64(sdf)), _d(m), _d(c), _d(I)), "mass_properties")
    return float(m[0]), c, I


def grid_layout(bbox_min, bbox_max, spacing, padding=2):
    """Origin and node counts of the grid Base::buildGrid lays over a bounding
    box (LevelSetObjectGenerator.h:122-183): padded by max(1, padding)
    spacings, snapped outwards to multiples of the spacing."""
    h = float(spacing)
    pad = max(1, int(padding)) * h
    lo = [h * math.floor((float(a) - pad) / h) for a in bbox_min]
    hi = [h * math.ceil((float(b) + pad) / h) for b in bbox_max]
    size = [int(math.floor((b - a) / h + 0.5)) + 1 for a, b in zip(lo, hi)]
    return np.array(lo), np.array(size, dtype=np.int32)


def levelset_grid(kind, param, origin, spacing, size, positive_inside=False, vertices=None, triangles=None,
                  device=-1, stream=None):
    """Signed-distance grid of a shape, evaluated on the GPU (Base::buildGrid,
    LevelSetObjectGenerator.h:122-224).  kind is one of SHAPES; param holds
    rx, ry, rz, ee, en (superellipsoid), radius (sphere), lx, ly, lz (box),
    A xyz, B xyz, radius (cylinder); a mesh takes vertices (n, 3) and
    triangles (m, 3).  Returns the nx*ny*nz values, x fastest."""
    sh = Shape()
    sh.kind = SHAPES[kind] if isinstance(kind, str) else int(kind)
    sh.positive_inside = 1 if positive_inside else 0
    p = _f64(param) if param is not None else np.zeros(0)
    for k in range(min(8, p.size)):
        sh.param[k] = p[k]
    keep = []
    if vertices is not None:
        v, t = _f64(vertices), _i32(triangles)
        keep += [v, t]
        sh.n_vertices, sh.vertices = v.size // 3, _d(v)
        sh.n_triangles, sh.triangles = t.size // 3, _i(t)
    n = _i32(size)
    out = np.empty(int(np.prod(n.astype(np.int64))), dtype=np.float64)
    _check(lib().fundem_levelset_grid(int(device), stream, C.byref(sh), _d(_f64(origin, 3)), float(spacing), _i(n),
                                      _d(out)), "levelset_grid")
    return out


def hash_sort(d_hash_ptr, n, num_cells, d_sorted_ptr, d_sorted_hash_ptr=None, stream=None):
    """fundem_hash_sort on device pointers (ints): stable order of 64-bit cell
    hashes, those outside [0, num_cells) last."""
    _check(lib().fundem_hash_sort(C.c_void_p(d_hash_ptr), int(n), int(num_cells), C.c_void_p(d_sorted_ptr),
                                  C.c_void_p(d_sorted_hash_ptr) if d_sorted_hash_ptr else None, stream), "hash_sort")


def prefix_sum(count, out=None, stream=None):
    """Inclusive prefix sum of a CUDA int32 tensor through the C ABI
    (the reference's buildPrefixSum); returns the output tensor."""
    import torch
    assert count.is_cuda and count.dtype == torch.int32 and count.is_contiguous()
    if out is None:
        out = torch.empty_like(count)
    _check(lib().fundem_prefix_sum(out.data_ptr(), count.data_ptr(), count.numel(), stream), "prefix_sum")
    return out


def _rot(q, v):
    qv = np.asarray(q[1:], float)
    t = 2.0 * np.cross(qv, v)
    return v + t * q[0] + np.cross(qv, t)


class Simulation:
    """One level-set DEM simulation on one GPU."""

    def __init__(self, device=0, stream=None, precision=FP64, records=True):
        self.L = lib()
        h = C.c_void_p()
        self._check(self.L.fundem_create(C.byref(h), int(device), stream), "create")
        self.h = h
        self._check(self.L.fundem_set_precision(self.h, int(precision)), "set_precision")
        self._check(self.L.fundem_set_records(self.h, int(bool(records))), "set_records")
        self.gravity = np.array([0.0, 0.0, -9.81])
        self.dt = 1e-6

    def _check(self, r, what=""):
        if r != 0:
            h = getattr(self, "h", None)
            detail = self.L.fundem_last_error(h).decode() if h else ""
            msg = lib().fundem_status_string(r).decode()
            raise FundemError(f"{what}: {msg} ({r})" + (f": {detail}" if detail else ""))

    def close(self):
        if getattr(self, "h", None):
            self.L.fundem_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------------ build
    @classmethod
    def from_scenario(cls, sc, device=0, precision=FP64, records=True, setup=True, stream=None):
        """Register a Scenario exactly as the reference API receives it:
        materials, geometries (explicit mass, or density through the
        addParticleCluster centroid handling, LSSolver.h:125-165), particles,
        walls, wall motion, bonds and periodicity."""
        s = cls(device=device, stream=stream, precision=precision, records=records)
        for (kn, ks, mu, e) in sc.particle_materials:
            s.add_material(False, kn, ks, mu, e)
        for (mu, e) in sc.wall_materials:
            s.add_material(True, 0.0, 0.0, mu, e)
        pos = np.array(sc.particles.pos, dtype=np.float64, copy=True)
        for gi, g in enumerate(sc.particle_geometries):
            if g.density is None:
                s.add_geometry(False, g.mass, g.inertia, g.origin, g.spacing, g.size, g.sdf, g.nodes)
            else:
                m, c, I = mass_properties(g.density, g.origin, g.spacing, g.size, g.sdf)
                s.add_geometry(False, m, I, np.asarray(g.origin, float) - c, g.spacing, g.size, g.sdf,
                               np.asarray(g.nodes, float) - c)
                for i in np.nonzero(sc.particles.geo == gi)[0]:
                    pos[i] = pos[i] + _rot(sc.particles.quat[i], c)
        for g in sc.wall_geometries:
            s.add_geometry(True, 0.0, None, g.origin, g.spacing, g.size, g.sdf, g.nodes)
        P = sc.particles
        s.add_objects(False, pos, P.vel, P.angvel, P.quat, P.mat, P.geo)
        W = sc.walls
        if len(W):
            s.add_objects(True, W.pos, W.vel, W.angvel, W.quat, W.mat, W.geo)
        for (idx, v, w) in sc.wall_motion:
            s.set_wall_motion(idx, v, w)
        B = sc.bonds
        if len(B):
            s.add_bonds(B.master, B.slave, B.point, B.normal, B.radius, B.length, B.young, B.poisson,
                        B.tensile, B.cohesion, B.friction)
        s.set_periodic(sc.periodic_x, sc.periodic_y)
        if getattr(sc, "periodic_sector", False):
            s.set_periodic_sector(True)
        if getattr(sc, "inertia", "reference") == "physical":
            s.set_inertia_mode(INERTIA_PHYSICAL)
        s.gravity = np.asarray(sc.gravity, float)
        s.dt = float(sc.dt)
        if setup:
            s.setup(sc.domain_min, sc.domain_max)
        return s

    def add_material(self, wall, kn, ks, mu, e):
        i = C.c_int()
        self._check(self.L.fundem_add_material(self.h, int(wall), kn, ks, mu, e, C.byref(i)), "add_material")
        if not wall:
            self._n_pmat = max(getattr(self, "_n_pmat", 0), i.value + 1)
        return i.value

    # ------------------------------------------------------------------ adjoint
    def adjoint_begin(self, checkpoint_interval=500):
        """Start recording from the current state (after detect) for reverse-mode
        gradients; a checkpoint every `checkpoint_interval` steps."""
        self._check(self.L.fundem_adjoint_begin(self.h, int(checkpoint_interval)), "adjoint_begin")

    def adjoint_forward(self, nsteps, gravity=None, dt=None):
        g = self.gravity if gravity is None else np.asarray(gravity, float)
        dt = self.dt if dt is None else float(dt)
        self._check(self.L.fundem_adjoint_forward(self.h, int(nsteps), _d(_f64(g, 3)), dt), "adjoint_forward")

    def adjoint_backward(self, dl_dpos, dl_dvel):
        """Gradients of a loss with the given gradients on the final positions
        and velocities: (d/d initial velocities (n, 3), d/d per particle
        material (kn, ks, damping ratio, mu) (n_materials, 4))."""
        n = self.num(False)
        gv0 = np.zeros((n, 3))
        gp = np.zeros((getattr(self, "_n_pmat", 1), 4))
        self._check(self.L.fundem_adjoint_backward(self.h, _d(_f64(dl_dpos, 3 * n)), _d(_f64(dl_dvel, 3 * n)),
                                                   _d(gv0), _d(gp)), "adjoint_backward")
        return gv0, gp

    def adjoint_backward_rot(self, dl_dpos, dl_dvel, dl_dquat=None, dl_dangvel=None):
        """As adjoint_backward, with loss gradients on the final orientations
        (n, 4) and angular velocities (n, 3) of turning bodies: returns
        (d/d initial velocities, d/d initial angular velocities, d/d per
        particle material)."""
        n = self.num(False)
        gv0, gw0 = np.zeros((n, 3)), np.zeros((n, 3))
        gp = np.zeros((getattr(self, "_n_pmat", 1), 4))
        q = None if dl_dquat is None else _f64(dl_dquat, 4 * n)
        w = None if dl_dangvel is None else _f64(dl_dangvel, 3 * n)
        self._check(self.L.fundem_adjoint_backward_rot(self.h, _d(_f64(dl_dpos, 3 * n)), _d(_f64(dl_dvel, 3 * n)),
                                                       _d(q), _d(w), _d(gv0), _d(gw0), _d(gp)), "adjoint_backward_rot")
        return gv0, gw0, gp

    def adjoint_end(self):
        self._check(self.L.fundem_adjoint_end(self.h), "adjoint_end")

    def add_geometry(self, wall, mass, inertia, origin, spacing, size, sdf, nodes):
        i = C.c_int()
        nodes = _f64(nodes)
        inertia = None if inertia is None else _f64(inertia, 6)
        self._check(self.L.fundem_add_geometry(self.h, int(wall), float(mass), _d(inertia), _d(_f64(origin, 3)),
                                          float(spacing), _i(_i32(size)), _d(_f64(sdf)), nodes.size // 3,
                                          _d(nodes), C.byref(i)), "add_geometry")
        return i.value

    def add_objects(self, wall, pos, vel, angvel, quat, mat, geo):
        pos = _f64(pos)
        n = pos.size // 3
        self._check(self.L.fundem_add_objects(self.h, int(wall), n, _d(pos), _d(_f64(vel, 3 * n)),
                                         _d(_f64(angvel, 3 * n)), _d(_f64(quat, 4 * n)), _i(_i32(mat)),
                                         _i(_i32(geo))), "add_objects")

    def set_wall_motion(self, idx, vel, angvel):
        self._check(self.L.fundem_set_wall_motion(self.h, int(idx), _d(_f64(vel, 3)), _d(_f64(angvel, 3))),
               "set_wall_motion")

    def add_bonds(self, master, slave, point, normal, radius, length, young, poisson, tensile=None,
                  cohesion=None, friction=None):
        master = _i32(master)
        n = master.size
        z = np.zeros(n)
        self._check(self.L.fundem_add_bonds(self.h, n, _i(master), _i(_i32(slave)), _d(_f64(point, 3 * n)),
                                       _d(_f64(normal, 3 * n)), _d(_f64(radius, n)), _d(_f64(length, n)),
                                       _d(_f64(young, n)), _d(_f64(poisson, n)),
                                       _d(_f64(z if tensile is None else tensile, n)),
                                       _d(_f64(z if cohesion is None else cohesion, n)),
                                       _d(_f64(z if friction is None else friction, n))), "add_bonds")

    def set_periodic(self, x, y):
        self._check(self.L.fundem_set_periodic(self.h, int(bool(x)), int(bool(y))), "set_periodic")

    def set_periodic_sector(self, on=True):
        """Quarter-sector periodicity about the z axis through the domain's
        min corner (LSSolver::addPeriodicBoundarySector)."""
        self._check(self.L.fundem_set_periodic_sector(self.h, int(bool(on))), "set_periodic_sector")

    def set_inertia_mode(self, mode):
        """INERTIA_REFERENCE (the reference's inverse(): zero when
        |det I| < 1e-30) or INERTIA_PHYSICAL (scale-aware); takes effect at
        the next setup."""
        self._check(self.L.fundem_set_inertia_mode(self.h, int(mode)), "set_inertia_mode")

    def checkpoint_write(self, path):
        """Write the state a restart needs (objects, contact history, bonds)."""
        self._check(self.L.fundem_checkpoint_write(self.h, os.fsencode(path)), "checkpoint_write")

    def checkpoint_read(self, path):
        """Restore a checkpoint into a simulation with the same setup."""
        self._check(self.L.fundem_checkpoint_read(self.h, os.fsencode(path)), "checkpoint_read")

    def set_neighbour_list(self, mode):
        """-1: from the particle count, 0: off, 1: on."""
        self._check(self.L.fundem_set_neighbour_list(self.h, int(mode)), "set_neighbour_list")

    def set_pair_cache(self, mode, skin=0.0):
        """Pair cache of the particle-particle list: mode -1 (default, from
        8192 particles), 0 off, 1 on; skin <= 0 takes the default skin."""
        self._check(self.L.fundem_set_pair_cache(self.h, int(mode), float(skin)), "set_pair_cache")

    def set_wall_groups(self, first, count):
        """Per particle, the first wall and the wall count it may meet (a
        batch of simulations tiled into one); empty arrays remove them."""
        first, count = _i32(first), _i32(count)
        self._check(self.L.fundem_set_wall_groups(self.h, int(first.size), _i(first), _i(count)), "set_wall_groups")

    def pair_cache_stats(self):
        """(rebuilds, steps run with the cache, skin in metres)."""
        r, n, sk = C.c_longlong(), C.c_longlong(), C.c_double()
        self._check(self.L.fundem_pair_cache_stats(self.h, C.byref(r), C.byref(n), C.byref(sk)), "pair_cache_stats")
        return r.value, n.value, sk.value

    def set_precision(self, precision):
        """FP64 (the reference's arithmetic) or FP32_MIXED; may change between steps."""
        self._check(self.L.fundem_set_precision(self.h, int(precision)), "set_precision")

    def set_records(self, full):
        self._check(self.L.fundem_set_records(self.h, int(bool(full))), "set_records")

    # ------------------------------------------------------------------ run
    def setup(self, minb, maxb):
        self._check(self.L.fundem_setup(self.h, _d(_f64(minb, 3)), _d(_f64(maxb, 3))), "setup")

    def detect(self):
        self._check(self.L.fundem_detect(self.h), "detect")

    def detect_proximity(self, gap):
        self._check(self.L.fundem_detect_proximity(self.h, float(gap)), "detect_proximity")

    def step(self, n=1, dt=None, gravity=None):
        g = _f64(self.gravity if gravity is None else gravity, 3)
        self._check(self.L.fundem_step(self.h, int(n), _d(g), float(self.dt if dt is None else dt)), "step")

    def step_graph(self, n, dt=None, gravity=None):
        """n steps recorded once into a CUDA graph and replayed on later calls
        (for many small simulations on separate streams)."""
        g = _f64(self.gravity if gravity is None else gravity, 3)
        self._check(self.L.fundem_step_graph(self.h, int(n), _d(g), float(self.dt if dt is None else dt)),
                    "step_graph")

    def step_begin(self, dt=None, gravity=None):
        g = _f64(self.gravity if gravity is None else gravity, 3)
        self._check(self.L.fundem_step_begin(self.h, _d(g), float(self.dt if dt is None else dt)), "step_begin")

    def step_end(self, dt=None, gravity=None):
        g = _f64(self.gravity if gravity is None else gravity, 3)
        self._check(self.L.fundem_step_end(self.h, _d(g), float(self.dt if dt is None else dt)), "step_end")

    def sync(self):
        self._check(self.L.fundem_sync(self.h), "sync")

    # ------------------------------------------------------------------ state
    def num(self, wall=False):
        n = C.c_int()
        self._check(self.L.fundem_num_objects(self.h, int(wall), C.byref(n)), "num_objects")
        return n.value

    def state(self, wall=False, out=None):
        """Object state as host arrays; `out` may supply the six arrays
        (C-contiguous float64, (n, 3) and (n, 4) for quat), for example in
        page-locked memory, and is filled in place."""
        n = self.num(wall)
        if out is None:
            out = {k: np.zeros((n, 3)) for k in ("pos", "vel", "angvel", "force", "torque")}
            out["quat"] = np.zeros((n, 4))
        else:
            for k, v in out.items():
                if not (v.dtype == np.float64 and v.flags.c_contiguous and v.shape == (n, 4 if k == "quat" else 3)):
                    raise ValueError(f"state(out=...): {k} must be a C-contiguous float64 array of shape "
                                     f"({n}, {4 if k == 'quat' else 3})")
        self._check(self.L.fundem_get_objects(self.h, int(wall), _d(out.get("pos")), _d(out.get("vel")),
                                              _d(out.get("angvel")), _d(out.get("quat")), _d(out.get("force")),
                                              _d(out.get("torque"))), "get_objects")
        return out

    def set_state(self, wall=False, pos=None, vel=None, angvel=None, quat=None, force=None, torque=None):
        n = self.num(wall)
        f = lambda a, k: None if a is None else _f64(a, n * k)
        self._check(self.L.fundem_set_objects(self.h, int(wall), _d(f(pos, 3)), _d(f(vel, 3)), _d(f(angvel, 3)),
                                         _d(f(quat, 4)), _d(f(force, 3)), _d(f(torque, 3))), "set_objects")

    def device_view(self, wall=False):
        v = DeviceView()
        self._check(self.L.fundem_device_view_get(self.h, int(wall), C.byref(v)), "device_view")
        return v

    def num_contacts(self, kind=PP):
        n = C.c_longlong()
        self._check(self.L.fundem_num_contacts(self.h, int(kind), C.byref(n)), "num_contacts")
        return n.value

    def num_pairs(self, kind=PP):
        n = C.c_longlong()
        self._check(self.L.fundem_num_pairs(self.h, int(kind), C.byref(n)), "num_pairs")
        return n.value

    def contacts(self, kind=PP):
        n = self.num_contacts(kind)
        c = dict(master=np.zeros(n, np.int32), slave=np.zeros(n, np.int32), point=np.zeros((n, 3)),
                 normal=np.zeros((n, 3)), overlap=np.zeros(n), spring=np.zeros((n, 3)), en=np.zeros(n),
                 es=np.zeros(n))
        if n:
            self._check(self.L.fundem_get_contacts(self.h, int(kind), _i(c["master"]), _i(c["slave"]), _d(c["point"]),
                                              _d(c["normal"]), _d(c["overlap"]), _d(c["spring"]), _d(c["en"]),
                                              _d(c["es"])), "get_contacts")
        return c

    def set_contacts(self, kind, node, partner, spring):
        node = _i32(node)
        self._check(self.L.fundem_set_contacts(self.h, int(kind), node.size, _i(node), _i(_i32(partner)),
                                          _d(_f64(spring, 3 * node.size))), "set_contacts")

    def bonds(self):
        n = C.c_int()
        self._check(self.L.fundem_num_bonds(self.h, C.byref(n)), "num_bonds")
        n = n.value
        act, pt, en = np.zeros(n, np.int32), np.zeros((n, 3)), np.zeros((n, 6))
        if n:
            self._check(self.L.fundem_get_bonds(self.h, _i(act), _d(pt), _d(en)), "get_bonds")
        return dict(activated=act, point=pt, un=en[:, 0], us=en[:, 1], ub=en[:, 2], ut=en[:, 3], sn=en[:, 4],
                    ss=en[:, 5])

    def set_bond_activation(self, act):
        self._check(self.L.fundem_set_bond_activation(self.h, _i(_i32(act))), "set_bond_activation")

    def geometry(self, geo, wall=False):
        r, im, I, Ii = np.zeros(1), np.zeros(1), np.zeros(6), np.zeros(6)
        self._check(self.L.fundem_get_geometry(self.h, int(wall), int(geo), _d(r), _d(im), _d(I), _d(Ii)), "geometry")
        return dict(radius=float(r[0]), inv_mass=float(im[0]), inertia=I, inv_inertia=Ii)

    def grid(self, wall=False):
        mn, mx, inv = np.zeros(3), np.zeros(3), np.zeros(3)
        sz = np.zeros(3, np.int32)
        self._check(self.L.fundem_get_grid(self.h, int(wall), _d(mn), _d(mx), _d(inv), _i(sz)), "grid")
        return dict(min=mn, max=mx, inv_cell=inv, size=sz)

    def set_profiling(self, on, counters=False):
        """Kernel-group timers (on) and narrow-phase work counters (counters).
        With the timers on, plain steps run every stage on the simulation's
        stream (the same results bit for bit), so each group's time is its
        own."""
        self._check(self.L.fundem_set_profiling(self.h, int(bool(on)) | (2 if counters else 0)), "set_profiling")

    def kernel_times(self):
        """{group: (milliseconds, intervals)} since the last call."""
        out = {}
        for name, k in TIMERS.items():
            ms, n = C.c_double(), C.c_longlong()
            self._check(self.L.fundem_kernel_time(self.h, k, C.byref(ms), C.byref(n)), "kernel_time")
            out[name] = (ms.value, n.value)
        return out

    def work_counters(self):
        """(pairs, clusters examined, clusters kept, node contacts, exact node
        tests of the selection, slots given the exact predicate by the cached
        predicate pass, slots it skipped by the slot bound) since the last
        call."""
        b = (C.c_ulonglong * 2)()
        self._check(self.L.fundem_slot_counters(self.h, b), "slot_counters")
        a = (C.c_ulonglong * 5)()
        self._check(self.L.fundem_work_counters(self.h, a), "work_counters")
        return tuple(int(x) for x in a) + tuple(int(x) for x in b)

    def set_launch_shape(self, select=0, probe=0, contact=0, sums=0):
        """Blocks per SM of the narrow phase's selection, predicate pass,
        contact-law pass and pair sums (0: default)."""
        a = (C.c_int * 4)(int(select), int(probe), int(contact), int(sums))
        self._check(self.L.fundem_set_launch_shape(self.h, a), "set_launch_shape")

    def launch_shape(self):
        a = (C.c_int * 4)()
        self._check(self.L.fundem_get_launch_shape(self.h, a), "launch_shape")
        return tuple(int(x) for x in a)

    def status_word(self):
        w = C.c_uint()
        self._check(self.L.fundem_status_word(self.h, C.byref(w)), "status_word")
        return w.value

    def status_word_to(self, address):
        """Enqueue a copy of the status word to a host address (page-locked
        memory: the copy does not stall the host; the word is there after
        sync())."""
        self._check(self.L.fundem_status_word(self.h, C.cast(C.c_void_p(int(address)), C.POINTER(C.c_uint))),
                    "status_word")

    def launch_count(self):
        n = C.c_longlong()
        self._check(self.L.fundem_launch_count(self.h, C.byref(n)), "launch_count")
        return n.value
