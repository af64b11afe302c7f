"""Reverse-mode (adjoint) gradients of the oracle's timestep: the FP64 CPU
reference adjoint.

Test infrastructure: only tests import this module.  The forward pass drives
the oracle (fundem_oracle.c) through its step in pieces, as oracle/tangent.py
does, and records at every step, for every contact, the local Jacobian of
(force on A, new sliding spring) with respect to (node offset from the
partner, contact velocity, previous spring, kn, ks, damping ratio, friction)
-- thirteen inputs, evaluated with forward-mode duals along the oracle's
state by the same contact evaluation as the tangent -- and, for every active
bond, the Jacobian of its force with respect to the bond vector.  The
backward pass then sweeps the steps last to first:

  Fbar_{n+1} += vbar_{n+1} dt / (2 m)                    (second half-kick)
  for each contact: g = J^T (Fbar_A - Fbar_B, Sbar_new)
      xbar_A += g_rel, xbar_B -= g_rel, vhbar_A += g_vc, vhbar_B -= g_vc
      (walls and a particle's own periodic image: no partner term; the
      image: no offset or velocity term), Sbar_prev[history slot] += g_S,
      material adjoints += g_params x their weights
  bonds: xbar_i += J^T (Fbar_i - Fbar_j), xbar_j -= the same
  vhbar += vbar_{n+1} + xbar dt,  vbar_n = vhbar,  Fbar_n = vhbar dt / (2 m)

The whole run is held in memory (no checkpoints): small cases only.  Its
gradients are those of the frozen-topology step, the same derivative the
tangent computes direction by direction.
"""
import numpy as np

from . import oracle as O
from .tangent import Dual, TangentRun, V3, dsqrt, dwhere, const, rotation, v3


class ReverseRun(TangentRun):
    """Oracle run of a scenario recorded for a reverse sweep.  step(T) runs
    and records; gradients(dl_dpos, dl_dvel) returns (d L / d initial
    velocities (n, 3), d L / d material parameters (n_materials, 4): kn, ks,
    damping ratio, friction) for L = sum(dl_dpos * x_T) + sum(dl_dvel * v_T)."""

    ND = 13  # rel 3, vc 3, previous spring 3, kn, ks, damping ratio, friction

    def __init__(self, sc):
        super().__init__(sc, [])
        assert not self.turning, "the reverse reference differentiates translating bodies only"
        self.tape = []

    def _step(self):
        o = self.o
        o.front()
        active = o.bonds()["activated"].copy() if len(self.bond_L0) else np.zeros(0, np.int32)
        o.detect_and_force()
        P, W = o.state(), o.state(wall=True)
        rec = {"contacts": [], "bonds": None}
        lists = {}
        for kind in self.kinds:
            c = o.contacts(kind)
            S = self._contact_setup(kind, c, P, W)
            if S is not None:
                rec["contacts"].append(self._local(S, kind))
            lists[kind] = (self._keys(c), c["spring"], np.zeros((0, len(c["master"]), 3)))
            rec.setdefault("nslots", {})[kind] = len(c["master"])
        self.lists = lists
        if len(self.bond_L0):
            rec["bonds"] = self._bond_jacobians(active, P)
        o.half_kick()
        self.tape.append(rec)

    def _local(self, S, kind):
        """The 13-input Jacobian of every contact of one list."""
        m, nd = S.m, self.ND
        eye = np.eye(nd)

        def seed(val, first):
            return v3(val, np.stack([np.broadcast_to(eye[:, first + k][:, None], (nd, m)) for k in range(3)], axis=2))

        rel = seed(S.gp - S.rj, 0)
        vc = seed(S.vc_val, 3)
        keys_prev, spr_prev, _ = self.lists[kind]
        has, hc = S.hist >= 0, np.where(S.hist >= 0, S.hist, 0)
        sp_val = np.where(has[:, None], spr_prev[hc] if len(spr_prev) else 0.0, 0.0)
        sprev = seed(sp_val, 6)
        par = [Dual(v, np.broadcast_to(eye[:, 9 + k][:, None], (nd, m)).copy())
               for k, v in enumerate((S.kn, S.ks, S.diss, S.mu))]
        F, snew, ok, _, _ = self._contact_eval(S, rel, vc, sprev, *par)
        J = np.concatenate([F.derivs(), snew.derivs()], axis=2)  # (13, m, 6)
        J[:, ~ok, :] = 0.0
        return {"kind": kind, "A": S.A, "j": S.j, "wall": S.wall, "react": S.react, "hist": S.hist, "J": J,
                "w": np.stack([S.w_kn, S.w_ks, S.w_diss, S.w_mu])}  # (4, np_dirs, m)

    def _bond_jacobians(self, active, P):
        on = np.nonzero(active != 0)[0]
        if len(on) == 0:
            return None
        b, f = self.bond_b[on], self.bond_f[on]
        i = np.asarray(self.sc.bonds.master, np.int64)[on]
        j = np.asarray(self.sc.bonds.slave, np.int64)[on]
        Ri, Rj = rotation(P["quat"][i]), rotation(P["quat"][j])
        rbi = P["pos"][i] + np.einsum("nab,nb->na", Ri, f[:, 3])
        rbj = P["pos"][j] + np.einsum("nab,nb->na", Rj, f[:, 7])
        dn = np.einsum("nab,nb->na", Rj, f[:, 4]) - np.einsum("nab,nb->na", Ri, f[:, 0])
        nb = len(on)
        rij = v3(rbi - rbj, np.stack([np.broadcast_to(np.eye(3)[:, k][:, None], (3, nb)) for k in range(3)], axis=2))
        D = dsqrt(rij.dot(rij))
        ok = D.v > 1e-20
        Ds = dwhere(ok, D, const(np.ones_like(D.v), 3))
        e = V3(-rij.x / Ds, -rij.y / Ds, -rij.z / Ds)
        dnv = v3(dn, np.zeros((3, nb, 3)))
        F = e.scale(b[:, 0] * (D - self.bond_L0[on])) + (dnv - e.scale(dnv.dot(e))).scale(b[:, 1] / (2.0 * Ds))
        J = F.derivs()  # (3 inputs, nb, 3 outputs)
        J[:, ~ok, :] = 0.0
        return {"i": i, "j": j, "J": J}

    def gradients(self, dl_dpos, dl_dvel):
        n, dt = self.n, float(self.sc.dt)
        half = np.where(self.inv_mass != 0.0, 0.5 * dt * self.inv_mass, 0.0)[:, None]
        xb = np.array(dl_dpos, float).reshape(n, 3).copy()
        vb = np.array(dl_dvel, float).reshape(n, 3).copy()
        Feb = np.zeros((n, 3))  # adjoint of the forces reaching the next step's first half-kick
        pgrad = np.zeros(self.np_dirs)
        Sb = {}  # spring adjoints of the current step's slots, per kind
        for t in range(len(self.tape) - 1, -1, -1):
            rec = self.tape[t]
            Fb = Feb + vb * half
            vhb = vb.copy()
            Sb_prev = {}
            prev = self.tape[t - 1]["nslots"] if t > 0 else None
            for L in rec["contacts"]:
                kind, A, j, react, J = L["kind"], L["A"], L["j"], L["react"], L["J"]
                m = len(A)
                fb = Fb[A] - np.where(react[:, None], Fb[np.where(L["wall"], A, j)], 0.0)
                sb = Sb.get(kind, np.zeros((m, 3)))
                g = np.einsum("kmo,mo->km", J, np.concatenate([fb, sb], axis=1))  # (13, m)
                move = L["wall"] | react  # a particle's own image: no offset or velocity term
                gx, gv = (g[0:3] * move).T, (g[3:6] * move).T
                np.add.at(xb, A, gx)
                np.add.at(vhb, A, gv)
                if not L["wall"]:
                    np.add.at(xb, j[react], -gx[react])
                    np.add.at(vhb, j[react], -gv[react])
                has = L["hist"] >= 0
                if t > 0 and has.any():
                    sp = Sb_prev.setdefault(kind, np.zeros((prev.get(kind, 0), 3)))
                    np.add.at(sp, L["hist"][has], g[6:9, has].T)
                pgrad += np.einsum("pdm,pm->d", L["w"], g[9:13])
            if rec["bonds"] is not None:
                B = rec["bonds"]
                fb = Fb[B["i"]] - Fb[B["j"]]
                g = np.einsum("kmo,mo->mk", B["J"], fb)
                np.add.at(xb, B["i"], g)
                np.add.at(xb, B["j"], -g)
            vh = vhb + dt * xb
            vb = vh
            Feb = vh * half
            Sb = Sb_prev
        return vb, pgrad.reshape(self.nmat, 4)
