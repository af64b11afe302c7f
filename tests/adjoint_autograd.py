"""torch.autograd wrapper of the adjoint, for the test harness only.

`DEMRun.apply(v0, params, backend, steps)` runs `steps` steps from initial
velocities `v0` (n, 3) with per-material parameters `params`
(n_materials, 4: kn, ks, damping ratio, friction) and returns the final
positions and velocities; `backward` hands their gradients to the backend's
reverse sweep and returns the gradients of `v0` and `params`.  Two backends:

* `OracleBackend`: the FP64 CPU reference adjoint (oracle/reverse.py);
* `SimulationBackend`: the library's C-ABI pair fundem_adjoint_forward /
  fundem_adjoint_backward on the GPU.

Contact topology is frozen per step in both, so the gradients are those of
the frozen-topology step.
"""
import copy

import numpy as np
import torch


def scenario_with(sc, v0, params):
    """A copy of `sc` with initial velocities v0 and material parameters
    (kn, ks, damping ratio, friction) per particle material."""
    s2 = copy.deepcopy(sc)
    s2.particles.vel = np.array(v0, float).reshape(len(s2.particles), 3)
    mats = []
    for kn, ks, zeta, mu in np.asarray(params, float).reshape(-1, 4):
        e = float(np.exp(-np.pi * zeta / np.sqrt(1.0 - zeta * zeta)))
        mats.append((float(kn), float(ks), float(mu), e))
    s2.particle_materials = mats
    return s2


def material_parameters(sc):
    """(n_materials, 4) kn, ks, damping ratio, friction of a scenario."""
    out = []
    for kn, ks, mu, e in sc.particle_materials:
        lr = np.log(e)
        out.append((kn, ks, -lr / np.sqrt(lr * lr + np.pi * np.pi), mu))
    return np.array(out, float)


class OracleBackend:
    def __init__(self, sc):
        self.sc = sc
        self.run = None

    def forward(self, v0, params, steps):
        from oracle import reverse
        if self.run is not None:
            self.run.close()
        self.run = reverse.ReverseRun(scenario_with(self.sc, v0, params))
        self.run.step(steps)
        st = self.run.o.state()
        return st["pos"], st["vel"]

    def backward(self, dl_dpos, dl_dvel):
        return self.run.gradients(dl_dpos, dl_dvel)


class SimulationBackend:
    def __init__(self, sc, fundem, checkpoint_interval=16):
        self.sc, self.F, self.K = sc, fundem, checkpoint_interval
        self.sim = None

    def forward(self, v0, params, steps):
        if self.sim is not None:
            self.sim.adjoint_end()
            self.sim.close()
        s = self.F.Simulation.from_scenario(scenario_with(self.sc, v0, params), records=False)
        s.detect()
        s.adjoint_begin(self.K)
        s.adjoint_forward(steps)
        self.sim = s
        st = s.state()
        return st["pos"], st["vel"]

    def backward(self, dl_dpos, dl_dvel):
        return self.sim.adjoint_backward(dl_dpos, dl_dvel)


class DEMRun(torch.autograd.Function):
    @staticmethod
    def forward(ctx, v0, params, backend, steps):
        x, v = backend.forward(v0.detach().cpu().numpy(), params.detach().cpu().numpy(), int(steps))
        ctx.backend = backend
        return torch.from_numpy(np.array(x, np.float64)), torch.from_numpy(np.array(v, np.float64))

    @staticmethod
    def backward(ctx, gx, gv):
        g_v0, g_p = ctx.backend.backward(gx.detach().cpu().numpy().astype(np.float64),
                                         gv.detach().cpu().numpy().astype(np.float64))
        return torch.from_numpy(np.array(g_v0, np.float64)), torch.from_numpy(np.array(g_p, np.float64)), None, None
