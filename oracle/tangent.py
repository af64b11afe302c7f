"""Forward-mode (tangent-linear) derivative of the oracle's timestep.

Test infrastructure: only tests import this module.  It is the FP64 CPU
reference for the GPU adjoint (fundem_adjoint_*), computed by a different
method (forward mode, vectorised over derivative directions) in a different
code base (numpy over the oracle's run).

The oracle (fundem_oracle.c) is driven through its step in pieces --
half-kick and drift (orc_front), detection and forces (orc_detect_and_force),
half-kick (orc_half_kick) -- and next to its values this module carries the
derivatives of positions, velocities, forces and sliding springs along a set
of directions: one material's kn, ks, damping ratio or friction coefficient,
or a change of the initial velocities.  The derivative is the one an adjoint
of the frozen-topology step computes: the contact lists, history links,
stick/slip branches and bond breakage of each step are the oracle's.
Bodies may turn (nonzero inverse inertia): orientations, angular velocities
and torques then carry derivatives too, through the world-frame inertia of
the kicks, the normalised quaternion step and the lever arms of the contact
torques; runs with turning bodies have no bonds (the GPU adjoint refuses
that combination as well).

Equations, following the reference step (LSSolver.h:1033-1107):
  v_h     = v_n + (F_n / m + g) dt / 2          (skipped when 1/m is zero)
  w_h     = w_n + I_w^-1 (T_n - w_n x I_w w_n) dt / 2,  I_w = R(q_n) I R(q_n)^T
            (particleIntegrationKernel.cu:3-32, myMat.h:107-158)
  x_{n+1} = x_n + v_h dt
  q_{n+1} = normalise(q_n + (0, w_h dt / 2) (x) q_n)   (myQua.h:77-93)
  contacts (contactKernel.cu:46-291, contactKernel.cuh:4-77): for a node of
    A at gp inside partner B (centre r_B, orientation q_B),
      rel = gp - r_B, local = R(q_B)^T rel, trilinear SDF value phi and the
      gradient with the int-truncated x weight
      (LSParticleContactDetectionKernel.cuh:4-77), n = R(q_B) grad / |grad|,
      overlap = -phi, contact point c = gp + n overlap / 2
      (LSParticleContactDetectionKernel.cu:268-281),
      v_c = v_A + w_A x (c - r_A) - v_B - w_B x (c - r_B),
      linear spring-dashpot normal force, sliding spring with Coulomb limit,
      torques (c - r_A) x F on A and (c - r_B) x (-F) on B, where the node
      gp = x_A + R(q_A) node moves with A's orientation;
  bonds (contactKernel.cuh:138-199): F = B1 (D - L0) e
    + B2 / (2 D) (dn - (dn . e) e), e = -(rb_i - rb_j) / D;
  v_{n+1} = v_h + (F_{n+1} / m + g) dt / 2,  w_{n+1} likewise from T_{n+1}
            at q_{n+1}.
The damping ratio comes from the restitution coefficient as the reference
forms it (contactKernel.cuh:49-51), in double precision here.  The effective
parameters of a contact (harmonic-mean stiffness, minimum friction and
restitution, contactKernel.cu:100-110, 190-200) carry their derivatives to
the material that sets them; where a minimum is taken between two equal
values the derivative goes to the particle's own material.
"""
import numpy as np

from . import oracle as O
from .oracle import OracleWorld, prepared_particles

PARAMS = ("kn", "ks", "damping", "mu")


# ---------------------------------------------------------------------------
# dual numbers over numpy: value (n,), derivatives (ND, n)
# ---------------------------------------------------------------------------
class Dual:
    __slots__ = ("v", "d")
    __array_ufunc__ = None  # ndarray (op) Dual defers to Dual's reflected operators

    def __init__(self, v, d):
        self.v = v
        self.d = d

    def _lift(self, o):
        if isinstance(o, Dual):
            return o
        o = np.asarray(o, float)
        return Dual(np.broadcast_to(o, self.v.shape), np.zeros_like(self.d))

    def __add__(self, o):
        o = self._lift(o)
        return Dual(self.v + o.v, self.d + o.d)

    __radd__ = __add__

    def __sub__(self, o):
        o = self._lift(o)
        return Dual(self.v - o.v, self.d - o.d)

    def __rsub__(self, o):
        return self._lift(o) - self

    def __neg__(self):
        return Dual(-self.v, -self.d)

    def __mul__(self, o):
        o = self._lift(o)
        return Dual(self.v * o.v, self.d * o.v + self.v * o.d)

    __rmul__ = __mul__

    def __truediv__(self, o):
        o = self._lift(o)
        q = self.v / o.v
        return Dual(q, (self.d - q * o.d) / o.v)

    def __rtruediv__(self, o):
        return self._lift(o) / self


def dsqrt(a):
    v = np.sqrt(a.v)
    g = np.where(v > 0.0, 0.5 / np.where(v > 0.0, v, 1.0), 0.0)
    return Dual(v, a.d * g)


def dwhere(mask, a, b):
    return Dual(np.where(mask, a.v, b.v), np.where(mask, a.d, b.d))


def const(v, nd):
    v = np.asarray(v, float)
    return Dual(v, np.zeros((nd,) + v.shape))


def deriv(d):
    """A dual with value zero and the given derivatives (ND, n)."""
    return Dual(np.zeros(d.shape[1:]), d)


class V3:
    """Three duals."""
    __slots__ = ("x", "y", "z")

    def __init__(self, x, y, z):
        self.x, self.y, self.z = x, y, z

    def __add__(self, o):
        return V3(self.x + o.x, self.y + o.y, self.z + o.z)

    def __sub__(self, o):
        return V3(self.x - o.x, self.y - o.y, self.z - o.z)

    def scale(self, s):
        return V3(s * self.x, s * self.y, s * self.z)

    def dot(self, o):
        return self.x * o.x + self.y * o.y + self.z * o.z

    def where(self, mask, o):
        return V3(dwhere(mask, self.x, o.x), dwhere(mask, self.y, o.y), dwhere(mask, self.z, o.z))

    def value(self):
        return np.stack([self.x.v, self.y.v, self.z.v], axis=1)

    def derivs(self):
        return np.stack([self.x.d, self.y.d, self.z.d], axis=2)  # (ND, n, 3)


def v3(val, der):
    """V3 from values (n, 3) and derivatives (ND, n, 3)."""
    return V3(Dual(val[:, 0], der[:, :, 0]), Dual(val[:, 1], der[:, :, 1]), Dual(val[:, 2], der[:, :, 2]))


def cross_const(w, a):
    """w x a for constant vectors w (n, 3) and a V3 a."""
    return V3(w[:, 1] * a.z - w[:, 2] * a.y, w[:, 2] * a.x - w[:, 0] * a.z, w[:, 0] * a.y - w[:, 1] * a.x)


def rotation(q):
    """Rotation matrices (n, 3, 3) of unit quaternions (scalar first)."""
    q0, q1, q2, q3 = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    R = np.empty((len(q), 3, 3))
    R[:, 0, 0] = 1 - 2 * (q2 * q2 + q3 * q3)
    R[:, 0, 1] = 2 * (q1 * q2 - q0 * q3)
    R[:, 0, 2] = 2 * (q1 * q3 + q0 * q2)
    R[:, 1, 0] = 2 * (q1 * q2 + q0 * q3)
    R[:, 1, 1] = 1 - 2 * (q1 * q1 + q3 * q3)
    R[:, 1, 2] = 2 * (q2 * q3 - q0 * q1)
    R[:, 2, 0] = 2 * (q1 * q3 - q0 * q2)
    R[:, 2, 1] = 2 * (q2 * q3 + q0 * q1)
    R[:, 2, 2] = 1 - 2 * (q1 * q1 + q2 * q2)
    return R


def dquat(q, dq):
    """Quaternions (n, 4) with derivatives (ND, n, 4) as four duals."""
    return [Dual(q[:, c], dq[:, :, c]) for c in range(4)]


def drotation(qd):
    """Rotation matrix (rows of duals) of dual unit quaternions, as rotation()."""
    q0, q1, q2, q3 = qd
    return [[1.0 - 2.0 * (q2 * q2 + q3 * q3), 2.0 * (q1 * q2 - q0 * q3), 2.0 * (q1 * q3 + q0 * q2)],
            [2.0 * (q1 * q2 + q0 * q3), 1.0 - 2.0 * (q1 * q1 + q3 * q3), 2.0 * (q2 * q3 - q0 * q1)],
            [2.0 * (q1 * q3 - q0 * q2), 2.0 * (q2 * q3 + q0 * q1), 1.0 - 2.0 * (q1 * q1 + q2 * q2)]]


def matvec(M, a):
    return V3(M[0][0] * a.x + M[0][1] * a.y + M[0][2] * a.z,
              M[1][0] * a.x + M[1][1] * a.y + M[1][2] * a.z,
              M[2][0] * a.x + M[2][1] * a.y + M[2][2] * a.z)


def vcross(a, b):
    """a x b for two V3s."""
    return V3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x)


def sym3(I6):
    """Symmetric tensors stored (xx, yy, zz, xy, xz, yz), (n, 6) -> (n, 3, 3)."""
    I6 = np.asarray(I6, float).reshape(-1, 6)
    xx, yy, zz, xy, xz, yz = I6.T
    return np.stack([np.stack([xx, xy, xz], 1), np.stack([xy, yy, yz], 1), np.stack([xz, yz, zz], 1)], 1)


def world_tensor(R, I):
    """R I R^T for a dual rotation R and constant tensors I (n, 3, 3)."""
    T = [[sum(R[a][c] * I[:, c, d] for c in range(3)) for d in range(3)] for a in range(3)]
    return [[sum(T[a][d] * R[b][d] for d in range(3)) for b in range(3)] for a in range(3)]


def dquat_integrate(qd, w, dt):
    """The quaternion step of myQua.h:77-93 on duals: q + (0, w dt / 2) (x) q,
    normalised."""
    q0, q1, q2, q3 = qd
    vx, vy, vz = w.x * (0.5 * dt), w.y * (0.5 * dt), w.z * (0.5 * dt)
    s0 = q0 + ((-q1) * vx - q2 * vy - q3 * vz)
    s1 = q1 + (q0 * vx + q3 * vy - q2 * vz)
    s2 = q2 + ((-q3) * vx + q0 * vy + q1 * vz)
    s3 = q3 + (q2 * vx - q1 * vy + q0 * vz)
    inv = 1.0 / dsqrt(s0 * s0 + s1 * s1 + s2 * s2 + s3 * s3)
    return [s0 * inv, s1 * inv, s2 * inv, s3 * inv]


def _stack(parts):
    """Derivatives of a list of duals, stacked on a last axis: (ND, n, k)."""
    return np.stack([p.d for p in parts], axis=2)


class _GeoTable:
    """SDF grids of a geometry set, concatenated."""

    def __init__(self, geos):
        self.origin = np.array([np.asarray(g["origin"], float) for g in geos]).reshape(-1, 3)
        self.inv_h = np.array([1.0 / float(g["spacing"]) for g in geos])
        self.size = np.array([np.asarray(g["size"], np.int64) for g in geos]).reshape(-1, 3)
        sdfs = [np.asarray(g["sdf"], float).ravel() for g in geos]
        self.off = np.concatenate([[0], np.cumsum([len(s) for s in sdfs])[:-1]]).astype(np.int64)
        self.sdf = np.concatenate(sdfs) if sdfs else np.zeros(0)


def _diss(e):
    lr = np.log(e)
    return -lr / np.sqrt(lr * lr + np.pi * np.pi)


class TangentRun:
    """The oracle's run of a scenario with derivatives along
    4 * (particle materials) parameter directions (kn, ks, damping ratio and
    friction of each material, in that order) followed by one direction per
    initial-velocity change in `vel_dirs` (each an (N, 3) array), then one
    per initial angular-velocity change in `angvel_dirs`.

    After step(T), directional(dl_dpos, dl_dvel, dl_dquat, dl_dangvel) gives
    d L / d direction for L = sum(dl_dpos * x_T) + sum(dl_dvel * v_T)
    + sum(dl_dquat * q_T) + sum(dl_dangvel * w_T): the four material
    gradients and the projections of d L / d v_0 and d L / d w_0 on the
    directions, which an adjoint gives in one backward sweep."""

    def __init__(self, sc, vel_dirs=(), angvel_dirs=()):
        assert not getattr(sc, "periodic_sector", False), "sector images are not differentiated"
        self.sc = sc
        self.o = OracleWorld.from_scenario(sc)
        geos, _ = prepared_particles(sc)
        self.pgeo = _GeoTable(geos)
        self.wgeo = _GeoTable([dict(origin=g.origin, spacing=g.spacing, size=g.size, sdf=g.sdf)
                               for g in sc.wall_geometries])
        P = sc.particles
        self.n = n = len(P)
        self.geo = np.asarray(P.geo, np.int64)
        self.mat = np.asarray(P.mat, np.int64)
        counts = np.array([len(geos[g]["nodes"]) for g in self.geo])
        self.node_pid = np.repeat(np.arange(n), counts)
        self.inv_mass = np.array([self.o.geometry(int(g))["inv_mass"] for g in self.geo])
        gp = [self.o.geometry(g) for g in range(len(geos))]
        self.inertia = sym3([g["inertia"] for g in gp])
        self.inv_inertia = sym3([g["inv_inertia"] for g in gp])
        self.turning = bool(np.any(self.inv_inertia[np.unique(self.geo)]))
        assert not (self.turning and len(sc.bonds)), "bonds between turning bodies are not differentiated"
        # body-frame node offsets, indexed by global boundary-node index
        self.node_local = np.concatenate([np.asarray(geos[g]["nodes"], float).reshape(-1, 3) for g in self.geo])
        # materials as the oracle stores them (orc_add_material's clamps)
        pm = np.array(sc.particle_materials, float).reshape(-1, 4)
        self.kn = np.where(pm[:, 0] > 0, pm[:, 0], 0.0)
        self.ks = np.where(pm[:, 1] > 0, pm[:, 1], 0.0)
        self.mu = np.where(pm[:, 2] > 0, pm[:, 2], 0.0)
        self.e = np.where((pm[:, 3] > 0) & (pm[:, 3] < 1), pm[:, 3], 1.0)
        wm = np.array(sc.wall_materials, float).reshape(-1, 2)
        self.wmu = np.where(wm[:, 0] > 0, wm[:, 0], 0.0)
        self.we = np.where((wm[:, 1] > 0) & (wm[:, 1] < 1), wm[:, 1], 1.0)
        self.wall_geo = np.asarray(sc.walls.geo, np.int64)
        self.wall_mat = np.asarray(sc.walls.mat, np.int64)
        self.nmat = len(pm)
        self.np_dirs = 4 * self.nmat
        self.nd = nd = self.np_dirs + len(vel_dirs) + len(angvel_dirs)
        self.dx = np.zeros((nd, n, 3))
        self.dv = np.zeros((nd, n, 3))
        self.dw = np.zeros((nd, n, 3))
        self.dq = np.zeros((nd, n, 4))
        for k, r in enumerate(vel_dirs):
            self.dv[self.np_dirs + k] = np.asarray(r, float).reshape(n, 3)
        for k, r in enumerate(angvel_dirs):
            self.dw[self.np_dirs + len(vel_dirs) + k] = np.asarray(r, float).reshape(n, 3)
        self.dF = np.zeros((nd, n, 3))
        self.dT = np.zeros((nd, n, 3))
        self.max_quat_dev = 0.0     # recomputed orientations against the oracle's
        grid = self.o.grid()
        span = grid["max"] - grid["min"]
        # ghost images sit one period above the domain (ghost_positions)
        self.shift = {O.GX: np.array([span[0], 0.0, 0.0]), O.GY: np.array([0.0, span[1], 0.0]),
                      O.GXY: np.array([span[0], span[1], 0.0])}
        self.kinds = [O.PP, O.PW] + ([O.GX] if sc.periodic_x else []) + ([O.GY] if sc.periodic_y else []) + \
                     ([O.GXY] if (sc.periodic_x and sc.periodic_y) else [])
        self.max_overlap_dev = 0.0  # recomputed overlaps against the oracle's
        self.max_spring_dev = 0.0   # recomputed springs against the oracle's
        self.bond_b, self.bond_f = self.o.bond_params()
        self.bond_L0 = np.asarray(sc.bonds.length, float) if len(sc.bonds) else np.zeros(0)
        self.o.initial_detect()
        self.lists = {}
        for k in self.kinds:
            c = self.o.contacts(k)
            self.lists[k] = (self._keys(c), c["spring"], np.zeros((nd, len(c["master"]), 3)))

    @staticmethod
    def _keys(c):
        return {(int(m), int(s)): i for i, (m, s) in enumerate(zip(c["master"], c["slave"]))}

    # -- steps ----------------------------------------------------------------
    def step(self, steps=1):
        for _ in range(steps):
            self._step()

    def _kick_w(self, st, dq, dw, dT, h):
        """Derivative of the angular half-kick w + I_w^-1 (T - w x I_w w) h,
        I_w = R(q) I R(q)^T (particleIntegrationKernel.cu:3-32), at the
        state `st`; bodies with zero inverse mass take no kick."""
        if not self.turning:
            return dw
        R = drotation(dquat(st["quat"], dq))
        w = v3(st["angvel"], dw)
        Iw = world_tensor(R, self.inertia[self.geo])
        Ii = world_tensor(R, self.inv_inertia[self.geo])
        acc = matvec(Ii, v3(st["torque"], dT) - vcross(w, matvec(Iw, w)))
        kicked = (self.inv_mass != 0.0)[None, :, None]
        return np.where(kicked, dw + h * acc.derivs(), dw)

    def _step(self):
        o, dt = self.o, float(self.sc.dt)
        kick = np.where(self.inv_mass != 0.0, 0.5 * dt * self.inv_mass, 0.0)[None, :, None]
        st0 = o.state() if self.turning else None
        dvh = self.dv + self.dF * kick
        dwh = self._kick_w(st0, self.dq, self.dw, self.dT, 0.5 * dt)
        self.dx = self.dx + dvh * dt
        o.front()
        if self.turning:
            st1 = o.state()
            qn = dquat_integrate(dquat(st0["quat"], self.dq), v3(st1["angvel"], dwh), dt)
            self.dq = _stack(qn)
            qv = np.stack([c.v for c in qn], axis=1)
            self.max_quat_dev = max(self.max_quat_dev, float(np.abs(qv - st1["quat"]).max()))
        active = o.bonds()["activated"].copy() if len(self.bond_L0) else np.zeros(0, np.int32)
        o.detect_and_force()
        P, W = o.state(), o.state(wall=True)
        dF = np.zeros_like(self.dF)
        dT = np.zeros_like(self.dT)
        self.lists = {kind: self._contacts(kind, o.contacts(kind), P, W, dvh, dwh, dF, dT) for kind in self.kinds}
        if len(self.bond_L0):
            self._bonds(active, P, dF)
        o.half_kick()
        self.dv = dvh + dF * kick
        self.dw = self._kick_w(P, self.dq, dwh, dT, 0.5 * dt)
        self.dF = dF
        self.dT = dT

    def _contacts(self, kind, c, P, W, dvh, dwh, dF, dT):
        nd = self.nd
        S = self._contact_setup(kind, c, P, W)
        if S is None:
            return ({}, c["spring"], np.zeros((nd, 0, 3)))
        A, j, wall, react, m = S.A, S.j, S.wall, S.react, S.m
        # the node's offset from A's centre, R(q_A) node, turns with A
        RA = drotation(dquat(P["quat"][A], self.dq[:, A, :]))
        armA = matvec(RA, v3(self.node_local[c["master"]], np.zeros((nd, m, 3))))
        S.armA_d = armA.derivs()
        # partner orientation: particles (and their images) turn, walls do not
        S.dqB = np.zeros((nd, m, 4)) if wall else self.dq[:, j, :]
        # rel = gp - r_B: derivative dx_A + d(R(q_A) node) - dx_B (dx terms
        # cancel for a particle's own image); walls do not move with the
        # parameters
        rel = v3(S.gp - S.rj, self.dx[:, A, :] - (0.0 if wall else self.dx[:, j, :]) + S.armA_d)
        dvc = dvh[:, A, :] - (0.0 if wall else dvh[:, j, :])
        if self.turning:
            dvc = dvc + np.cross(dwh[:, A, :], (S.point - S.ri)[None])
            if not wall:
                dvc = dvc - np.cross(dwh[:, j, :], (S.point - S.rj)[None])
        vc = v3(S.vc_val, dvc)
        pad = np.zeros((nd - self.np_dirs, m))
        Kn = Dual(S.kn, np.vstack([S.w_kn, pad]))
        Ks = Dual(S.ks, np.vstack([S.w_ks, pad]))
        Diss = Dual(S.diss, np.vstack([S.w_diss, pad]))
        Mu = Dual(S.mu, np.vstack([S.w_mu, pad]))
        # the previous spring: first match of (node, partner) in the previous list
        _, spr_prev, dS_prev = self.lists[kind]
        has, hc = S.hist >= 0, np.where(S.hist >= 0, S.hist, 0)
        sp_val = np.where(has[:, None], spr_prev[hc] if len(spr_prev) else 0.0, 0.0)
        sp_der = np.where(has[None, :, None], dS_prev[:, hc, :] if dS_prev.shape[1] else 0.0, 0.0)
        F, snew, ok, TA, TB = self._contact_eval(S, rel, vc, v3(sp_val, sp_der), Kn, Ks, Diss, Mu)
        Fd = np.where(ok[None, :, None], F.derivs(), 0.0)
        if self.turning:
            np.add.at(dT, (slice(None), A), np.where(ok[None, :, None], TA, 0.0))
            if not wall:
                TBd = np.where(ok[None, :, None], TB, 0.0)
                np.add.at(dT, (slice(None), j[react]), TBd[:, react])
        Sd = np.where(ok[None, :, None], snew.derivs(), 0.0)
        Sv = np.where(ok[:, None], snew.value(), 0.0)
        scale = max(float(np.abs(c["spring"]).max()), 1e-300)
        self.max_spring_dev = max(self.max_spring_dev, float(np.abs(Sv - c["spring"]).max()) / scale)
        np.add.at(dF, (slice(None), A), Fd)
        if not wall:
            np.add.at(dF, (slice(None), j[react]), -Fd[:, react])
        return (self._keys(c), c["spring"], Sd)

    class _Contacts:
        """Values of one contact list at one step (see _contact_setup)."""

    def _contact_setup(self, kind, c, P, W):
        """Partners, state values, effective parameters and their weights on
        the material parameter directions (4 per material: kn, ks, damping
        ratio, friction), and history slots of the contacts of list `kind`
        (contactKernel.cu:46-291)."""
        m = len(c["master"])
        if m == 0:
            return None
        S = TangentRun._Contacts()
        S.m, S.kind = m, kind
        S.A = A = self.node_pid[c["master"]]
        S.j = j = c["slave"].astype(np.int64)
        S.wall = wall = kind == O.PW
        ghost = kind in self.shift
        point, normal, overlap = c["point"], c["normal"], c["overlap"]
        S.overlap = overlap
        S.gp = point - normal * (0.5 * overlap)[:, None]
        if wall:
            rj, vj, S.wj, S.qB = W["pos"][j], W["vel"][j], W["angvel"][j], W["quat"][j]
            S.G, S.geoB = self.wgeo, self.wall_geo[j]
        else:
            rj, vj, S.wj, S.qB = P["pos"][j], P["vel"][j], P["angvel"][j], P["quat"][j]
            if ghost:
                rj = rj + self.shift[kind]
            S.G, S.geoB = self.pgeo, self.geo[j]
        S.rj = rj
        S.point = point
        # a contact with a particle's own periodic image has no reaction
        S.react = np.zeros(m, bool) if wall else (j != A) if ghost else np.ones(m, bool)
        ri, vi = P["pos"][A], P["vel"][A]
        S.ri = ri
        S.wi = P["angvel"][A]
        S.vc_val = (vi + np.cross(S.wi, point - ri)) - (vj + np.cross(S.wj, point - rj))
        # effective parameters and their weights on the material directions
        mi = self.mat[A]
        kni, ksi, mui, ei = self.kn[mi], self.ks[mi], self.mu[mi], self.e[mi]
        im_i = self.inv_mass[A]
        w = [np.zeros((self.np_dirs, m)) for _ in range(4)]
        cols = np.arange(m)
        if wall:
            mw = self.wall_mat[j]
            kn, ks = kni, ksi
            mu = np.minimum(mui, self.wmu[mw])
            res = np.minimum(ei, self.we[mw])
            meff = np.where(im_i > 0, 1.0 / np.where(im_i > 0, im_i, 1.0), 0.0)
            w[0][4 * mi, cols] = 1.0
            w[1][4 * mi + 1, cols] = 1.0
            own_e, own_mu = ei <= self.we[mw], mui <= self.wmu[mw]
            w[2][4 * mi[own_e] + 2, cols[own_e]] = 1.0
            w[3][4 * mi[own_mu] + 3, cols[own_mu]] = 1.0
        else:
            mj = self.mat[j]
            knj, ksj = self.kn[mj], self.ks[mj]
            okn, oks = (kni > 0) & (knj > 0), (ksi > 0) & (ksj > 0)
            skn, sks = np.where(okn, kni + knj, 1.0), np.where(oks, ksi + ksj, 1.0)
            kn = np.where(okn, kni * knj / skn, 0.0)
            ks = np.where(oks, ksi * ksj / sks, 0.0)
            np.add.at(w[0], (4 * mi, cols), np.where(okn, knj * knj / skn ** 2, 0.0))
            np.add.at(w[0], (4 * mj, cols), np.where(okn, kni * kni / skn ** 2, 0.0))
            np.add.at(w[1], (4 * mi + 1, cols), np.where(oks, ksj * ksj / sks ** 2, 0.0))
            np.add.at(w[1], (4 * mj + 1, cols), np.where(oks, ksi * ksi / sks ** 2, 0.0))
            im_j = self.inv_mass[j]
            ssum = im_i + im_j
            meff = np.where((im_i > 0) | (im_j > 0), 1.0 / np.where(ssum != 0, ssum, 1.0), 0.0)
            res = np.minimum(ei, self.e[mj])
            mu = np.minimum(mui, self.mu[mj])
            w[2][4 * np.where(ei <= self.e[mj], mi, mj) + 2, cols] = 1.0
            w[3][4 * np.where(mui <= self.mu[mj], mi, mj) + 3, cols] = 1.0
        S.kn = np.broadcast_to(np.asarray(kn, float), (m,)).copy()
        S.ks = np.broadcast_to(np.asarray(ks, float), (m,)).copy()
        S.diss = _diss(res)
        S.mu = np.asarray(mu, float)
        S.meff = meff
        S.w_kn, S.w_ks, S.w_diss, S.w_mu = w
        keys = self.lists[kind][0]
        S.hist = np.array([keys.get((int(a), int(b)), -1) for a, b in zip(c["master"], c["slave"])], np.int64)
        return S

    def _contact_eval(self, S, rel, vc, sprev, Kn, Ks, Diss, Mu):
        """Force on A and new sliding spring of each contact as duals of the
        seeded node offset `rel`, contact velocity `vc` (its dependence on the
        contact point is added here), previous spring and parameters; also
        the mask of contacts that carry a force and the derivatives of the
        torques on A and B (None when no body turns)."""
        if self.turning:
            R = drotation(dquat(S.qB, S.dqB))
        else:
            Rc = rotation(S.qB)
            R = [[Rc[:, a, b] for b in range(3)] for a in range(3)]
        lx = rel.x * R[0][0] + rel.y * R[1][0] + rel.z * R[2][0]
        ly = rel.x * R[0][1] + rel.y * R[1][1] + rel.z * R[2][1]
        lz = rel.x * R[0][2] + rel.y * R[1][2] + rel.z * R[2][2]
        G = S.G
        org, ih, sz, off = G.origin[S.geoB], G.inv_h[S.geoB], G.size[S.geoB], G.off[S.geoB]
        gx, gy, gz = (lx - org[:, 0]) * ih, (ly - org[:, 1]) * ih, (lz - org[:, 2]) * ih
        i0 = np.floor(gx.v).astype(np.int64)
        j0 = np.floor(gy.v).astype(np.int64)
        k0 = np.floor(gz.v).astype(np.int64)
        inside = (i0 >= 0) & (j0 >= 0) & (k0 >= 0) & (i0 < sz[:, 0] - 1) & (j0 < sz[:, 1] - 1) & \
                 (k0 < sz[:, 2] - 1)
        i0, j0, k0 = np.where(inside, i0, 0), np.where(inside, j0, 0), np.where(inside, k0, 0)
        sx, sxy = sz[:, 0], sz[:, 0] * sz[:, 1]
        base = off + k0 * sxy + j0 * sx + i0
        p = [G.sdf[base + d] for d in (0, 1)] + [G.sdf[base + sx + d] for d in (0, 1)] + \
            [G.sdf[base + sxy + d] for d in (0, 1)] + [G.sdf[base + sxy + sx + d] for d in (0, 1)]
        fx, fy, fz = gx - i0, gy - j0, gz - k0
        ux, uy, uz = 1.0 - fx, 1.0 - fy, 1.0 - fz
        phi = ((p[0] * ux + p[1] * fx) * uy + (p[2] * ux + p[3] * fx) * fy) * uz + \
              ((p[4] * ux + p[5] * fx) * uy + (p[6] * ux + p[7] * fx) * fy) * fz
        ov = -phi
        dev = np.abs(ov.v - S.overlap) / np.maximum(np.abs(S.overlap), 1e-300)
        self.max_overlap_dev = max(self.max_overlap_dev, float(np.max(np.where(inside, dev, 0.0))))
        # gradient with the x weight truncated to the cell's x = 0 face
        ggx = (p[1] - p[0]) * (uy * uz) + (p[3] - p[2]) * (fy * uz) + (p[5] - p[4]) * (uy * fz) + \
              (p[7] - p[6]) * (fy * fz)
        ggy = (p[2] - p[0]) * uz + (p[6] - p[4]) * fz
        ggz = (p[4] - p[0]) * uy + (p[6] - p[2]) * fy
        nw = V3(ggx * R[0][0] + ggy * R[0][1] + ggz * R[0][2],
                ggx * R[1][0] + ggy * R[1][1] + ggz * R[1][2],
                ggx * R[2][0] + ggy * R[2][1] + ggz * R[2][2])
        nl = dsqrt(nw.dot(nw))
        n = V3(nw.x / nl, nw.y / nl, nw.z / nl)
        # contact velocity: c - r_A moves with n overlap / 2, c - r_B with rel
        # and n overlap / 2
        h = n.scale(0.5 * ov)
        hd = V3(deriv(h.x.d), deriv(h.y.d), deriv(h.z.d))
        reld = V3(deriv(rel.x.d), deriv(rel.y.d), deriv(rel.z.d))
        if getattr(S, "armA_d", None) is not None:
            vc = vc + cross_const(S.wi, v3(np.zeros((S.m, 3)), S.armA_d))
        vc = vc + cross_const(S.wi, hd) - cross_const(S.wj, reld + hd)
        F, snew = self._law(sprev, vc, n, ov, Kn, Ks, Diss, Mu, S.meff, float(self.sc.dt))
        TA = TB = None
        if self.turning:
            # lever arms c - r_A and c - r_B: values from the oracle's contact
            # point, derivatives through the node's turn, rel and n ov / 2
            armA = v3(S.point - S.ri, S.armA_d + h.derivs())
            armB = v3(S.point - S.rj, rel.derivs() + h.derivs())
            TA = vcross(armA, F).derivs()
            TB = vcross(armB, F.scale(-1.0)).derivs()
        return F, snew, inside & (ov.v > 0.0), TA, TB

    @staticmethod
    def _law(sprev, vc, n, ov, kn, ks, diss, mu, m, dt):
        """contactKernel.cuh:36-77 with integrateSlidingSpring, :4-34."""
        nd = kn.d.shape[0]
        one = const(np.ones_like(kn.v), nd)
        cn = 2.0 * diss * dsqrt(kn * m)
        vn = n.scale(vc.dot(n))
        fn = n.scale(kn * ov) - vn.scale(cn)
        cs = 2.0 * diss * dsqrt(ks * m)
        vs = vc - vn
        p1 = sprev - n.scale(sprev.dot(n))
        ap1 = dsqrt(p1.dot(p1))
        big = ap1.v > 1e-20
        p1 = p1.scale(dsqrt(sprev.dot(sprev)) / dwhere(big, ap1, one)).where(big, p1)
        sp = p1 + vs.scale(dt)
        sf = sp.scale(-1.0 * ks) - vs.scale(cs)
        asf = dsqrt(sf.dot(sf))
        afn = dsqrt(fn.dot(fn))
        slip = (asf.v > 1e-20) & (asf.v > mu.v * afn.v)
        t = sf.scale(mu * afn / dwhere(slip, asf, one)) + vs.scale(cs)
        sp = t.scale(-1.0 / dwhere(ks.v != 0.0, ks, one)).where(slip, sp)
        on = (mu.v > 0.0) & (ks.v > 0.0)
        zero = const(np.zeros_like(kn.v), nd)
        sp = sp.where(on, V3(zero, zero, zero))
        F = fn + (sp.scale(-1.0 * ks) - vs.scale(cs))
        return F, sp

    def _bonds(self, active, P, dF):
        on = np.nonzero(active != 0)[0]
        if len(on) == 0:
            return
        b, f = self.bond_b[on], self.bond_f[on]
        i = np.asarray(self.sc.bonds.master, np.int64)[on]
        j = np.asarray(self.sc.bonds.slave, np.int64)[on]
        Ri, Rj = rotation(P["quat"][i]), rotation(P["quat"][j])
        rbi = P["pos"][i] + np.einsum("nab,nb->na", Ri, f[:, 3])
        rbj = P["pos"][j] + np.einsum("nab,nb->na", Rj, f[:, 7])
        dn = np.einsum("nab,nb->na", Rj, f[:, 4]) - np.einsum("nab,nb->na", Ri, f[:, 0])
        rij = v3(rbi - rbj, self.dx[:, i, :] - self.dx[:, j, :])
        D = dsqrt(rij.dot(rij))
        ok = D.v > 1e-20
        Ds = dwhere(ok, D, const(np.ones_like(D.v), self.nd))
        e = V3(-rij.x / Ds, -rij.y / Ds, -rij.z / Ds)
        dnv = v3(dn, np.zeros((self.nd, len(on), 3)))
        F = e.scale(b[:, 0] * (D - self.bond_L0[on])) + (dnv - e.scale(dnv.dot(e))).scale(b[:, 1] / (2.0 * Ds))
        Fd = np.where(ok[None, :, None], F.derivs(), 0.0)
        np.add.at(dF, (slice(None), i), Fd)
        np.add.at(dF, (slice(None), j), -Fd)

    # -- results --------------------------------------------------------------
    def directional(self, dl_dpos, dl_dvel, dl_dquat=None, dl_dangvel=None):
        """d L / d direction for L = sum(dl_dpos * x_T) + sum(dl_dvel * v_T)
        + sum(dl_dquat * q_T) + sum(dl_dangvel * w_T)."""
        out = np.einsum("dnc,nc->d", self.dx, dl_dpos) + np.einsum("dnc,nc->d", self.dv, dl_dvel)
        if dl_dquat is not None:
            out = out + np.einsum("dnc,nc->d", self.dq, dl_dquat)
        if dl_dangvel is not None:
            out = out + np.einsum("dnc,nc->d", self.dw, dl_dangvel)
        return out

    def close(self):
        self.o.close()
