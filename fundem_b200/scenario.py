"""Scenario construction for the level-set DEM timestep.

Builds the inputs of the hot path: shape templates (signed-distance grids plus
surface-node meshes), materials, particles, walls and bonds.  This is the
caller side of the timestep, restated from the reference's host helpers:

* superellipsoid implicit function and gradient
  (kernel/helper/LevelSetObjectGenerator.h:1265-1340)
* signed-distance-like grid value f/|grad f| (LevelSetObjectGenerator.h:196-216)
* icosphere surface mesh projected radially onto the superellipsoid
  (LevelSetObjectGenerator.h:1034-1199)
* plane walls as 2x2x2 linear SDF grids (apps/test/LSSphereBouncing.cpp:86-129)

Templates here are sampled on an exact n^3 lattice (32^3 by default) with
spacing max(semi-axis)/14, centred on the body origin; values are rounded to
float32 when requested, so the same numbers feed the FP32 and FP64 paths.
"""
from __future__ import annotations

import dataclasses
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

PI = 3.14159265358979323846


# ---------------------------------------------------------------------------
# surface meshes
# ---------------------------------------------------------------------------
def _normalize_rows(v: np.ndarray) -> np.ndarray:
    n2 = np.einsum("ij,ij->i", v, v)
    inv = 1.0 / np.sqrt(n2)
    return v * inv[:, None]


def _orient_outward(verts: np.ndarray, tris: np.ndarray) -> np.ndarray:
    """Swap the last two indices of triangles whose normal points inward
    (LevelSetObjectGenerator.h:1120-1140)."""
    v0, v1, v2 = verts[tris[:, 0]], verts[tris[:, 1]], verts[tris[:, 2]]
    centre = (v0 + v1 + v2) / 3.0
    fn = np.cross(v1 - v0, v2 - v0)
    flip = np.einsum("ij,ij->i", fn, centre) < 0.0
    out = tris.copy()
    out[flip, 1], out[flip, 2] = tris[flip, 2], tris[flip, 1]
    return out


def icosphere(level: int):
    """Unit icosphere: icosahedron refined `level` times by edge midpoints
    pushed to the sphere.  Vertex order is the order of first creation, which
    is what gives boundary nodes their indices."""
    g = 0.5 * (1.0 + np.sqrt(5.0))
    base = np.array([[-1, g, 0], [1, g, 0], [-1, -g, 0], [1, -g, 0],
                     [0, -1, g], [0, 1, g], [0, -1, -g], [0, 1, -g],
                     [g, 0, -1], [g, 0, 1], [-g, 0, -1], [-g, 0, 1]], dtype=np.float64)
    verts = [tuple(r) for r in _normalize_rows(base)]
    tris = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11],
                     [1, 5, 9], [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8],
                     [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9],
                     [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], dtype=np.int64)
    tris = _orient_outward(np.array(verts), tris)
    for _ in range(level):
        cache = {}
        new_tris = []

        def mid(a, b):
            lo, hi = (a, b) if a < b else (b, a)
            key = (lo, hi)
            if key in cache:
                return cache[key]
            va, vb = np.array(verts[lo]), np.array(verts[hi])
            m = 0.5 * (va + vb)
            m = m * (1.0 / np.sqrt(np.dot(m, m)))
            verts.append(tuple(m))
            cache[key] = len(verts) - 1
            return cache[key]

        for t in tris:
            i0, i1, i2 = (int(x) for x in t)
            i01, i12, i20 = mid(i0, i1), mid(i1, i2), mid(i2, i0)
            new_tris += [(i0, i01, i20), (i1, i12, i01), (i2, i20, i12), (i01, i12, i20)]
        tris = _orient_outward(np.array(verts), np.array(new_tris, dtype=np.int64))
    return np.array(verts, dtype=np.float64), tris


def superellipsoid_value_grad(p: np.ndarray, rx, ry, rz, ee, en):
    """Implicit value and gradient (LevelSetObjectGenerator.h:1265-1340)."""
    irx, iry, irz = 1.0 / rx, 1.0 / ry, 1.0 / rz
    nx, ny, nz = np.abs(p[..., 0] * irx), np.abs(p[..., 1] * iry), np.abs(p[..., 2] * irz)
    exy, ez, outer = 2.0 / ee, 2.0 / en, ee / en
    xt, yt = np.power(nx, exy), np.power(ny, exy)
    s = xt + yt
    f = np.power(s, outer) + np.power(nz, ez) - 1.0
    eps = 1e-30
    ss, snx, sny, snz = (np.maximum(a, eps) for a in (s, nx, ny, nz))
    som1 = np.power(ss, outer - 1.0)
    sgn = lambda a: np.where(a >= 0.0, 1.0, -1.0)
    dsdx = exy * np.power(snx, exy - 1.0) * sgn(p[..., 0]) * irx
    dsdy = exy * np.power(sny, exy - 1.0) * sgn(p[..., 1]) * iry
    g = np.stack([outer * som1 * dsdx, outer * som1 * dsdy,
                  ez * np.power(snz, ez - 1.0) * sgn(p[..., 2]) * irz], axis=-1)
    return f, g


def superellipsoid_nodes(rx, ry, rz, ee, en, level=3):
    """Surface nodes: icosphere directions scaled onto the surface
    (projectUnitDirectionToSuperellipsoid, LevelSetObjectGenerator.h:1003-1032)."""
    verts, tris = icosphere(level)
    l2 = np.einsum("ij,ij->i", verts, verts)
    d = verts * (1.0 / np.sqrt(l2))[:, None]
    xt = np.power(np.abs(np.abs(d[:, 0] / rx)), 2.0 / ee)
    yt = np.power(np.abs(np.abs(d[:, 1] / ry)), 2.0 / ee)
    zt = np.power(np.abs(np.abs(d[:, 2] / rz)), 2.0 / en)
    scale = np.power(np.abs(xt + yt), ee / en) + zt
    radial = np.power(scale, -0.5 * en)
    nodes = d * radial[:, None]
    tris = _orient_outward(nodes, tris)
    return nodes, tris


# ---------------------------------------------------------------------------
# geometry templates
# ---------------------------------------------------------------------------
@dataclass
class Geometry:
    """One shape template.  `sdf` is flattened x-fastest (index
    z*ny*nx + y*nx + x, myVec.h:232-235).  Particle geometries carry either an
    explicit mass/inertia (density None) or a density from which mass
    properties are computed (LSSolver.h:470-586)."""
    origin: np.ndarray
    spacing: float
    size: np.ndarray
    sdf: np.ndarray
    nodes: np.ndarray
    tris: np.ndarray
    mass: float = 0.0
    inertia: np.ndarray = field(default_factory=lambda: np.zeros(6))
    density: Optional[float] = None


def superellipsoid_template(rx, ry, rz, ee, en, n=32, cells_per_rmax=None, level=3,
                            float32=True, density=None, mass=None, inertia=None) -> Geometry:
    """Template on an n^3 lattice centred on the body origin.  The spacing is
    max(semi-axis)/14 at n = 32 and scales with n so the lattice always spans
    +-(31/28) max(semi-axis)."""
    rmax = max(rx, ry, rz)
    if cells_per_rmax is None:
        cells_per_rmax = 14.0 * (n - 1) / 31.0
    h = rmax / cells_per_rmax
    ax = (np.arange(n, dtype=np.float64) - 0.5 * (n - 1)) * h
    Z, Y, X = np.meshgrid(ax, ax, ax, indexing="ij")
    p = np.stack([X, Y, Z], axis=-1)
    f, g = superellipsoid_value_grad(p, rx, ry, rz, ee, en)
    gn = np.sqrt(np.einsum("...i,...i->...", g, g))
    val = np.where(gn > 1e-12, f / np.where(gn > 1e-12, gn, 1.0),
                   np.where(f <= 0.0, -1.0, 1.0) * 0.5 * h)
    if float32:
        val = val.astype(np.float32).astype(np.float64)
    nodes, tris = superellipsoid_nodes(rx, ry, rz, ee, en, level)
    geo = Geometry(origin=np.array([ax[0]] * 3), spacing=h, size=np.array([n, n, n], dtype=np.int32),
                   sdf=val.reshape(-1).copy(), nodes=nodes, tris=tris.astype(np.int32))
    if density is not None:
        geo.density = float(density)
    elif mass is not None:
        geo.mass = float(mass)
        geo.inertia = np.asarray(inertia, dtype=np.float64)
    return geo


def sphere_template(radius, n=13, level=2, density=None, mass=None, inertia=None) -> Geometry:
    """Exact sphere SDF |p| - r on an n^3 lattice of spacing r/5
    (apps/test/LSSphereBouncing.cpp:26-45)."""
    h = radius / 5.0
    ax = (np.arange(n, dtype=np.float64) - 0.5 * (n - 1)) * h
    Z, Y, X = np.meshgrid(ax, ax, ax, indexing="ij")
    val = np.sqrt(X * X + Y * Y + Z * Z) - radius
    verts, tris = icosphere(level)
    geo = Geometry(origin=np.array([ax[0]] * 3), spacing=h, size=np.array([n, n, n], dtype=np.int32),
                   sdf=val.reshape(-1).copy(), nodes=verts * radius, tris=tris.astype(np.int32))
    if density is not None:
        geo.density = float(density)
    elif mass is not None:
        geo.mass = float(mass)
        geo.inertia = np.asarray(inertia, dtype=np.float64)
    return geo


def plane_wall_template(extent: float) -> Geometry:
    """Plane z = 0 (SDF = local z) on a 2x2x2 grid of spacing `extent`
    centred on the wall origin; four corner nodes."""
    h = float(extent)
    origin = np.array([-0.5 * h] * 3)
    vals = []
    for z in range(2):
        for y in range(2):
            for x in range(2):
                vals.append(origin[2] + z * h)
    c = 0.5 * h
    nodes = np.array([[-c, -c, 0.0], [c, -c, 0.0], [c, c, 0.0], [-c, c, 0.0]])
    tris = np.array([[0, 1, 2], [0, 2, 3]], dtype=np.int32)
    return Geometry(origin=origin, spacing=h, size=np.array([2, 2, 2], dtype=np.int32),
                    sdf=np.array(vals, dtype=np.float64), nodes=nodes, tris=tris)


# rotations taking the wall's local +z to an inward normal
_S = np.sqrt(0.5)
WALL_QUAT = {
    "+z": (1.0, 0.0, 0.0, 0.0), "-z": (0.0, 1.0, 0.0, 0.0),
    "+x": (_S, 0.0, _S, 0.0), "-x": (_S, 0.0, -_S, 0.0),
    "+y": (_S, -_S, 0.0, 0.0), "-y": (_S, _S, 0.0, 0.0),
}


def random_quaternions(rng: np.random.Generator, n: int) -> np.ndarray:
    """Uniform random unit quaternions (Shoemake's method), scalar first."""
    u1, u2, u3 = rng.random(n), rng.random(n), rng.random(n)
    s1, s2 = np.sqrt(1.0 - u1), np.sqrt(u1)
    a, b = 2.0 * PI * u2, 2.0 * PI * u3
    return np.stack([s2 * np.cos(b), s1 * np.sin(a), s1 * np.cos(a), s2 * np.sin(b)], axis=1)


# ---------------------------------------------------------------------------
# scenario container
# ---------------------------------------------------------------------------
@dataclass
class Objects:
    pos: np.ndarray
    vel: np.ndarray
    angvel: np.ndarray
    quat: np.ndarray
    mat: np.ndarray
    geo: np.ndarray

    @staticmethod
    def empty():
        z3 = np.zeros((0, 3))
        return Objects(z3, z3.copy(), z3.copy(), np.zeros((0, 4)), np.zeros(0, np.int32), np.zeros(0, np.int32))

    def __len__(self):
        return len(self.pos)


@dataclass
class Bonds:
    master: np.ndarray
    slave: np.ndarray
    point: np.ndarray
    normal: np.ndarray
    radius: np.ndarray
    length: np.ndarray
    young: np.ndarray
    poisson: np.ndarray
    tensile: np.ndarray
    cohesion: np.ndarray
    friction: np.ndarray

    @staticmethod
    def empty():
        z = np.zeros(0)
        return Bonds(np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros((0, 3)), np.zeros((0, 3)),
                     z, z.copy(), z.copy(), z.copy(), z.copy(), z.copy(), z.copy())

    def __len__(self):
        return len(self.master)


@dataclass
class Scenario:
    domain_min: np.ndarray
    domain_max: np.ndarray
    gravity: np.ndarray
    dt: float
    particle_materials: List[tuple]
    wall_materials: List[tuple]
    particle_geometries: List[Geometry]
    wall_geometries: List[Geometry]
    particles: Objects
    walls: Objects
    wall_motion: List[tuple] = field(default_factory=list)   # (index, velocity, angular velocity)
    bonds: Bonds = field(default_factory=Bonds.empty)
    periodic_x: bool = False
    periodic_y: bool = False
    # quarter-sector periodicity about the z axis through domain_min
    # (LSSolver::addPeriodicBoundarySector)
    periodic_sector: bool = False
    # inverse-inertia rule: "reference" (|det I| < 1e-30 gives zero, so
    # mm-scale bodies never turn) or "physical" (scale-aware)
    inertia: str = "reference"
    name: str = "scenario"

    def copy(self) -> "Scenario":
        return dataclasses.replace(self)


# ---------------------------------------------------------------------------
# geometric queries used while building scenarios (numpy, host side)
# ---------------------------------------------------------------------------
def _rot(q, v):
    """Rotate v (..., 3) by unit quaternions q (..., 4)."""
    qv = q[..., 1:]
    t = 2.0 * np.cross(qv, v)
    return v + t * q[..., :1] + np.cross(qv, t)


def _rrot(v, q):
    qc = q.copy()
    qc[..., 1:] *= -1.0
    return _rot(qc, v)


def _trilinear(geo: Geometry, g: np.ndarray):
    """SDF value at grid coordinates g (..., 3); nan outside the grid."""
    nx, ny, nz = (int(s) for s in geo.size)
    i0 = np.floor(g).astype(np.int64)
    inside = np.all((i0 >= 0) & (i0 < np.array([nx - 1, ny - 1, nz - 1])), axis=-1)
    i0 = np.clip(i0, 0, np.array([nx - 2, ny - 2, nz - 2]))
    f = g - i0
    S = geo.sdf.reshape(nz, ny, nx)
    out = 0.0
    for dz in (0, 1):
        wz = f[..., 2] if dz else 1.0 - f[..., 2]
        for dy in (0, 1):
            wy = f[..., 1] if dy else 1.0 - f[..., 1]
            for dx in (0, 1):
                wx = f[..., 0] if dx else 1.0 - f[..., 0]
                out = out + S[i0[..., 2] + dz, i0[..., 1] + dy, i0[..., 0] + dx] * wx * wy * wz
    return np.where(inside, out, np.nan)


def min_surface_gap(geos, objs: Objects, pairs: np.ndarray, chunk=4096):
    """For each pair (i, j): the smallest SDF value of j sampled at i's nodes
    and of i at j's nodes, the midpoint across the gap at that node (world
    frame) and the unit centre-to-centre direction from j to i."""
    n = len(pairs)
    gap = np.full(n, np.inf)
    where = np.zeros((n, 3))
    normal = np.zeros((n, 3))
    for side in (0, 1):
        a_idx, b_idx = (pairs[:, 0], pairs[:, 1]) if side == 0 else (pairs[:, 1], pairs[:, 0])
        for s in range(0, n, chunk):
            sl = slice(s, min(n, s + chunk))
            ga, gb = objs.geo[a_idx[sl]], objs.geo[b_idx[sl]]
            for gA in np.unique(ga):
                for gB in np.unique(gb):
                    m = (ga == gA) & (gb == gB)
                    if not np.any(m):
                        continue
                    ia, ib = a_idx[sl][m], b_idx[sl][m]
                    GA, GB = geos[gA], geos[gB]
                    nodes = _rot(objs.quat[ia][:, None, :], GA.nodes[None, :, :]) + objs.pos[ia][:, None, :]
                    rel = nodes - objs.pos[ib][:, None, :]
                    loc = _rrot(rel, np.repeat(objs.quat[ib][:, None, :], GA.nodes.shape[0], axis=1))
                    g = (loc - GB.origin) / GB.spacing
                    phi = _trilinear(GB, g)
                    phi = np.where(np.isnan(phi), np.inf, phi)
                    k = np.argmin(phi, axis=1)
                    val = phi[np.arange(len(k)), k]
                    rows = np.nonzero(m)[0] + s
                    better = val < gap[rows]
                    rows_b = rows[better]
                    gap[rows_b] = val[better]
                    d = objs.pos[ia] - objs.pos[ib]
                    d = d / np.maximum(np.linalg.norm(d, axis=1, keepdims=True), 1e-300)
                    # midpoint across the gap: the sampled node moves half the
                    # gap toward the other body (along -d)
                    mid = nodes[np.arange(len(k)), k] - 0.5 * np.maximum(val, 0.0)[:, None] * d
                    where[rows_b] = mid[better]
                    normal[rows_b] = (d if side == 0 else -d)[better]
    return gap, where, normal


def candidate_pairs(pos: np.ndarray, radius: np.ndarray, margin=0.0):
    """All pairs (i<j) whose bounding spheres (plus margin) intersect,
    by a uniform cell grid."""
    n = len(pos)
    if n < 2:
        return np.zeros((0, 2), np.int64)
    cell = 2.0 * (radius.max() + margin)
    key = np.floor((pos - pos.min(axis=0)) / cell).astype(np.int64)
    dims = key.max(axis=0) + 3
    lin = ((key[:, 2] + 1) * dims[1] + (key[:, 1] + 1)) * dims[0] + (key[:, 0] + 1)
    order = np.argsort(lin, kind="stable")
    lin_sorted = lin[order]
    out = []
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                target = lin + (dz * dims[1] + dy) * dims[0] + dx
                lo = np.searchsorted(lin_sorted, target, "left")
                hi = np.searchsorted(lin_sorted, target, "right")
                cnt = hi - lo
                if cnt.max(initial=0) == 0:
                    continue
                rep_i = np.repeat(np.arange(n), cnt)
                starts = np.repeat(lo, cnt)
                offs = np.arange(cnt.sum()) - np.repeat(np.cumsum(cnt) - cnt, cnt)
                rep_j = order[starts + offs]
                keep = rep_i < rep_j
                out.append(np.stack([rep_i[keep], rep_j[keep]], axis=1))
    pairs = np.concatenate(out) if out else np.zeros((0, 2), np.int64)
    d = np.linalg.norm(pos[pairs[:, 0]] - pos[pairs[:, 1]], axis=1)
    keep = d <= radius[pairs[:, 0]] + radius[pairs[:, 1]] + 2 * margin
    pairs = pairs[keep]
    return pairs[np.lexsort((pairs[:, 1], pairs[:, 0]))]


def node_radius(geo: Geometry) -> float:
    return float(np.max(np.sqrt(np.einsum("ij,ij->i", geo.nodes, geo.nodes))))


def resolve_overlaps(rng, geos, objs: Objects, max_rounds=200, tries=24, tol=0.0):
    """Give every particle whose surface overlaps a neighbour a new
    orientation: `tries` random candidates are scored by the smallest gap to
    all bounding-sphere neighbours and the best is kept; repeat until no pair
    overlaps.  Returns the number of particles re-oriented."""
    radius = np.array([node_radius(geos[g]) for g in objs.geo])
    pairs = candidate_pairs(objs.pos, radius)
    if len(pairs) == 0:
        return 0
    changed = set()
    for _ in range(max_rounds):
        gap, _, _ = min_surface_gap(geos, objs, pairs)
        bad = pairs[gap <= tol]
        if len(bad) == 0:
            return len(changed)
        # one particle per bad pair, at most one fix per particle per round
        cand = np.unique(np.where(rng.random(len(bad)) < 0.5, bad[:, 0], bad[:, 1]))
        for i in cand:
            nb = pairs[(pairs[:, 0] == i) | (pairs[:, 1] == i)]
            qs = random_quaternions(rng, tries)
            best, best_q = -np.inf, None
            old = objs.quat[i].copy()
            for q in qs:
                objs.quat[i] = q
                g, _, _ = min_surface_gap(geos, objs, nb)
                m = g.min() if len(g) else np.inf
                if m > best:
                    best, best_q = m, q.copy()
            objs.quat[i] = best_q if best_q is not None else old
            changed.add(int(i))
    raise RuntimeError("could not resolve initial overlaps")


# ---------------------------------------------------------------------------
# scenario builders
# ---------------------------------------------------------------------------
def superellipsoid_templates(rng, count, lo=0.8e-3, hi=1.2e-3, n=32, level=3, density=2500.0,
                             exponents=(2.0, 4.0), explicit_mass=False):
    """`count` templates with semi-axes uniform in [lo, hi] and exponents from
    `exponents` (exponent 2/ee -> ee = 2/exponent)."""
    geos = []
    for _ in range(count):
        rx, ry, rz = rng.uniform(lo, hi, 3)
        ee = 2.0 / exponents[rng.integers(len(exponents))]
        en = 2.0 / exponents[rng.integers(len(exponents))]
        geos.append(superellipsoid_template(rx, ry, rz, ee, en, n=n, level=level, density=density))
    if explicit_mass:
        for g in geos:
            m, c, I = mass_properties(g.density, g.origin, g.spacing, g.size, g.sdf)
            g.origin = g.origin - c
            g.nodes = g.nodes - c
            g.mass, g.inertia, g.density = m, I, None
    return geos


def mass_properties(density, origin, h, size, sdf):
    """Mass, centroid and inertia from a smoothed Heaviside of phi/h with
    smoothing width 1.5 (LSSolver.h:503-565), vectorised."""
    nx, ny, nz = (int(s) for s in size)
    phi = sdf.reshape(nz, ny, nx) / h
    x = -phi / 1.5
    H = np.where(phi < -1.5, 1.0, np.where(phi > 1.5, 0.0, 0.5 * (1.0 + x + np.sin(PI * x) / PI)))
    mg = density * h * h * h
    mass = H.sum() * mg
    Z, Y, X = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    P = np.stack([origin[0] + X * h, origin[1] + Y * h, origin[2] + Z * h], axis=-1)
    c = (H[..., None] * P).reshape(-1, 3).sum(axis=0) * mg / mass
    r = P - c
    w = H * mg
    I = np.array([(w * (r[..., 1] ** 2 + r[..., 2] ** 2)).sum(), (w * (r[..., 0] ** 2 + r[..., 2] ** 2)).sum(),
                  (w * (r[..., 1] ** 2 + r[..., 0] ** 2)).sum(), -(w * r[..., 0] * r[..., 1]).sum(),
                  -(w * r[..., 0] * r[..., 2]).sum(), -(w * r[..., 1] * r[..., 2]).sum()])
    return mass, c, I


def box_walls(lo, hi, faces=("+z", "-z", "+x", "-x", "+y", "-y"), margin_frac=0.1):
    """Plane walls on the faces of the box [lo, hi] with inward normals.  One
    geometry per wall (extent covering the face) and wall centres on the face
    centres."""
    lo, hi = np.asarray(lo, float), np.asarray(hi, float)
    ext = float(np.max(hi - lo)) * (1.0 + margin_frac)
    c = 0.5 * (lo + hi)
    centres = {"+z": [c[0], c[1], lo[2]], "-z": [c[0], c[1], hi[2]], "+x": [lo[0], c[1], c[2]],
               "-x": [hi[0], c[1], c[2]], "+y": [c[0], lo[1], c[2]], "-y": [c[0], hi[1], c[2]]}
    geos, pos, quat = [], [], []
    for f in faces:
        geos.append(plane_wall_template(ext))
        pos.append(centres[f])
        quat.append(WALL_QUAT[f])
    n = len(faces)
    walls = Objects(np.array(pos, float), np.zeros((n, 3)), np.zeros((n, 3)), np.array(quat, float),
                    np.zeros(n, np.int32), np.arange(n, dtype=np.int32))
    return geos, walls


def lattice_positions(rng, n, box_lo, box_hi, pitch, jitter):
    box_lo, box_hi = np.asarray(box_lo, float), np.asarray(box_hi, float)
    counts = np.maximum(1, np.floor((box_hi - box_lo) / pitch).astype(int))
    if counts.prod() < n:
        raise ValueError(f"lattice {counts} holds {counts.prod()} < {n} particles")
    idx = np.arange(n)
    ix = idx % counts[0]
    iy = (idx // counts[0]) % counts[1]
    iz = idx // (counts[0] * counts[1])
    pos = box_lo + (np.stack([ix, iy, iz], axis=1) + 0.5) * pitch
    pos += rng.uniform(-jitter, jitter, size=pos.shape)
    return pos


def pour(n=1000, n_templates=4, seed=0, box=(20e-3, 20e-3, 40e-3), pitch=2.5e-3, jitter=0.05e-3,
         kn=1e4, kt_ratio=0.8, damping_ratio=0.3, friction=0.5, density=2500.0, dt=1e-6,
         grid_n=32, level=3, walls=True, resolve=True, explicit_mass=False, init_speed=0.0,
         restitution=None, name="pour"):
    """Small pour: superellipsoids on a jittered lattice in a box with six
    plane walls, random orientations, gravity -z."""
    rng = np.random.default_rng(seed)
    geos = superellipsoid_templates(rng, n_templates, n=grid_n, level=level, density=density,
                                    explicit_mass=explicit_mass)
    box_lo, box_hi = np.zeros(3), np.asarray(box, float)
    pos = lattice_positions(rng, n, box_lo, box_hi, pitch, jitter)
    geo = rng.integers(0, n_templates, n).astype(np.int32)
    if not explicit_mass:
        order = np.argsort(geo, kind="stable")
        geo = geo[order]
        pos = pos[order]
    quat = random_quaternions(rng, n)
    vel = rng.uniform(-1, 1, (n, 3)) * init_speed
    objs = Objects(pos, vel, np.zeros((n, 3)), quat, np.zeros(n, np.int32), geo)
    resampled = resolve_overlaps(rng, geos, objs) if resolve else 0
    e = restitution if restitution is not None else float(np.exp(-PI * damping_ratio / np.sqrt(1 - damping_ratio ** 2)))
    wall_geos, wall_objs = box_walls(box_lo, box_hi) if walls else ([], Objects.empty())
    margin = 2e-3
    sc = Scenario(domain_min=box_lo - margin, domain_max=box_hi + margin, gravity=np.array([0.0, 0.0, -9.81]),
                  dt=dt, particle_materials=[(kn, kt_ratio * kn, friction, e)],
                  wall_materials=[(friction, e)], particle_geometries=geos, wall_geometries=wall_geos,
                  particles=objs, walls=wall_objs, name=name)
    sc.resampled = resampled
    return sc


def bonded_periodic(n=512, n_templates=8, seed=1, footprint=None, pitch=2.4e-3, jitter=0.02e-3,
                    kn=1e4, kt_ratio=0.8, damping_ratio=0.3, friction=0.5, density=2500.0, dt=5e-7,
                    grid_n=32, level=3, bond_gap_frac=0.05, young=1e8, poisson=0.3, tensile=1e6,
                    bond_radius_frac=0.3, platen_speed=1.0, resolve=True, name="bonded_periodic"):
    """Periodic-in-x/y column on a floor wall with a moving top platen, bonds
    between particle pairs whose surface gap is below `bond_gap_frac` of the
    mean diameter."""
    rng = np.random.default_rng(seed)
    geos = superellipsoid_templates(rng, n_templates, n=grid_n, level=level, density=density)
    if footprint is None:
        side = int(np.ceil(np.sqrt(n / 4.0)))
        footprint = (side * pitch, side * pitch)
    fx, fy = footprint
    nx, ny = int(round(fx / pitch)), int(round(fy / pitch))
    nz = int(np.ceil(n / (nx * ny)))
    box_lo = np.zeros(3)
    box_hi = np.array([nx * pitch, ny * pitch, nz * pitch])
    pos = lattice_positions(rng, n, box_lo, box_hi + 1e-12, pitch, jitter)
    geo = rng.integers(0, n_templates, n).astype(np.int32)
    order = np.argsort(geo, kind="stable")
    geo, pos = geo[order], pos[order]
    quat = random_quaternions(rng, n)
    objs = Objects(pos, np.zeros((n, 3)), np.zeros((n, 3)), quat, np.zeros(n, np.int32), geo)
    resampled = resolve_overlaps(rng, geos, objs) if resolve else 0
    e = float(np.exp(-PI * damping_ratio / np.sqrt(1 - damping_ratio ** 2)))
    # floor and top platen; wall centres inside the domain (reference hashes
    # only objects whose centre lies in [min, max))
    top = box_hi[2] + 0.5 * pitch
    ext = float(max(box_hi[0], box_hi[1])) * 1.1
    wall_geos = [plane_wall_template(ext), plane_wall_template(ext)]
    c = 0.5 * box_hi
    walls = Objects(np.array([[c[0], c[1], 0.0], [c[0], c[1], top]]), np.zeros((2, 3)), np.zeros((2, 3)),
                    np.array([WALL_QUAT["+z"], WALL_QUAT["-z"]]), np.zeros(2, np.int32),
                    np.array([0, 1], np.int32))
    dom_lo = np.array([0.0, 0.0, -2e-3])
    dom_hi = np.array([box_hi[0], box_hi[1], top + 2e-3])
    # bonds
    radius = np.array([node_radius(geos[g]) for g in objs.geo])
    d_mean = 2.0 * float(np.mean([np.mean(np.sqrt(np.einsum("ij,ij->i", g.nodes, g.nodes))) for g in geos]))
    thr = bond_gap_frac * d_mean
    pairs = candidate_pairs(objs.pos, radius, margin=0.5 * thr)
    gap, where, normal = min_surface_gap(geos, objs, pairs)
    sel = gap < thr
    bp = pairs[sel]
    point = where[sel]
    nb = len(bp)
    L0 = np.linalg.norm(objs.pos[bp[:, 0]] - objs.pos[bp[:, 1]], axis=1)  # centre distance
    bonds = Bonds(bp[:, 0].astype(np.int32), bp[:, 1].astype(np.int32), point, normal[sel],
                  np.full(nb, bond_radius_frac * 0.5 * d_mean), L0, np.full(nb, young), np.full(nb, poisson),
                  np.full(nb, tensile), np.zeros(nb), np.zeros(nb))
    sc = Scenario(domain_min=dom_lo, domain_max=dom_hi, gravity=np.array([0.0, 0.0, -9.81]), dt=dt,
                  particle_materials=[(kn, kt_ratio * kn, friction, e)], wall_materials=[(friction, e)],
                  particle_geometries=geos, wall_geometries=wall_geos, particles=objs, walls=walls,
                  wall_motion=[(1, np.array([0.0, 0.0, -platen_speed]), np.zeros(3))], bonds=bonds,
                  periodic_x=True, periodic_y=True, name=name)
    sc.resampled = resampled
    return sc


def sphere_on_plane(radius=0.01, density=2000.0, height=1.0, collide_time=0.005, dt_frac=50.0):
    """The sphere-bouncing case (apps/test/LSSphereBouncing.cpp): one sphere
    dropped on a plane, e = 1, kn = m pi^2 / (2 t_c^2)."""
    m = (4.0 / 3.0) * PI * radius ** 3 * density
    I = 0.4 * m * radius * radius
    kn = 0.5 * m * PI * PI / (collide_time * collide_time)
    geo = sphere_template(radius, mass=m, inertia=[I, I, I, 0, 0, 0])
    # six-by-six latitude/longitude node set of the app
    nodes = []
    ns = 6
    for i in range(ns):
        for j in range(ns):
            th, ph = i * PI / (ns - 1), j * 2.0 * PI / ns
            nodes.append([radius * np.sin(th) * np.cos(ph), radius * np.sin(th) * np.sin(ph), radius * np.cos(th)])
    geo.nodes = np.array(nodes)
    geo.tris = np.zeros((0, 3), np.int32)
    plane_min, plane_max = np.array([-0.5, -0.5, 0.0]), np.array([0.5, 0.5, 0.0])
    wg = plane_wall_template(1.0)
    objs = Objects(np.array([[0.0, 0.0, height]]), np.zeros((1, 3)), np.zeros((1, 3)),
                   np.array([[1.0, 0, 0, 0]]), np.zeros(1, np.int32), np.zeros(1, np.int32))
    walls = Objects(np.zeros((1, 3)), np.zeros((1, 3)), np.zeros((1, 3)), np.array([[1.0, 0, 0, 0]]),
                    np.zeros(1, np.int32), np.zeros(1, np.int32))
    return Scenario(domain_min=plane_min - np.array([0, 0, height]), domain_max=plane_max + np.array([0, 0, height]),
                    gravity=np.array([0.0, 0.0, -9.81]), dt=collide_time / dt_frac,
                    particle_materials=[(kn, 0.0, 0.0, 1.0)], wall_materials=[(0.0, 1.0)],
                    particle_geometries=[geo], wall_geometries=[wg], particles=objs, walls=walls,
                    name="sphere_on_plane")
