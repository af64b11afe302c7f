"""Batched calibration: many independent simulations of uneven size on one GPU.

`TiledBatch` places every simulation in its own region of space inside one
Simulation (`tile`): each stage of the timestep is then one launch over all
simulations' particles, with the per-simulation parameters as a block of
materials (simulation i uses material i) and per-particle wall groups (each
particle meets only its own simulation's walls).  The adjoint of the tiled
run gives every simulation's parameter gradients at once.

`Batch` is the alternative with one CUDA stream per simulation, stepping in
chunks recorded once into a CUDA graph (fundem_step_graph); the chunk length
comes from `autotune_chunk`, which times candidate lengths on the batch.

`calibration_scenarios` builds the calibration sweep: pours with particle
counts log-uniform in [500, 20000], per-simulation kn log-uniform in
[5e3, 5e4], friction uniform in [0.2, 0.8] and damping ratio uniform in
[0.1, 0.5], the small pour's shapes, in boxes sized for a fill ratio of 0.4.

Over several GPUs (one process per GPU), `shard` splits the simulations
whole, largest first, and `run_sharded` runs each rank's share and gathers
the per-simulation results on every rank; the simulations exchange nothing
while they run.
"""
from __future__ import annotations

import time

import numpy as np

from . import Simulation
from . import scenario as S


def calibration_scenarios(n_sims=256, seed=1, n_min=500, n_max=20000, fill=0.4, dt=1e-6, templates=None,
                          jitter=0.02e-3):
    """(scenarios, parameters): parameters holds per simulation n, kn, mu,
    damping ratio and the fill ratio actually built (the box grows when a
    non-overlapping lattice of the particles does not fit at 0.4)."""
    rng = np.random.default_rng(seed)
    if templates is None:
        templates = S.superellipsoid_templates(np.random.default_rng(seed + 1000), 4, n=32, level=3,
                                               density=2500.0, explicit_mass=True)
    counts = np.exp(rng.uniform(np.log(n_min), np.log(n_max), n_sims)).astype(int)
    kn = np.exp(rng.uniform(np.log(5e3), np.log(5e4), n_sims))
    mu = rng.uniform(0.2, 0.8, n_sims)
    zeta = rng.uniform(0.1, 0.5, n_sims)
    vp = float(np.mean([g.mass / 2500.0 for g in templates]))
    pitch = 2.0 * max(S.node_radius(g) for g in templates) * 1.01
    scenarios, params = [], []
    for i in range(n_sims):
        n = int(counts[i])
        side = (n * vp / fill / 2.0) ** (1.0 / 3.0)   # square base, height twice the side
        while np.prod(np.floor(np.array([side, side, 2 * side]) / pitch)) < n:
            side *= 1.05
        hi = np.array([side, side, 2 * side])
        pos = S.lattice_positions(rng, n, np.zeros(3), hi, pitch, jitter)
        geo = rng.integers(0, len(templates), n).astype(np.int32)
        quat = S.random_quaternions(rng, n)
        objs = S.Objects(pos, np.zeros((n, 3)), np.zeros((n, 3)), quat, np.zeros(n, np.int32), geo)
        e = float(np.exp(-np.pi * zeta[i] / np.sqrt(1.0 - zeta[i] ** 2)))
        wall_geos, walls = S.box_walls(np.zeros(3), hi)
        margin = 2e-3
        sc = S.Scenario(domain_min=-margin * np.ones(3), domain_max=hi + margin,
                        gravity=np.array([0.0, 0.0, -9.81]), dt=dt,
                        particle_materials=[(float(kn[i]), 0.8 * float(kn[i]), float(mu[i]), e)],
                        wall_materials=[(float(mu[i]), e)], particle_geometries=templates,
                        wall_geometries=wall_geos, particles=objs, walls=walls, name=f"calibration_{i}")
        scenarios.append(sc)
        params.append(dict(n=n, kn=float(kn[i]), mu=float(mu[i]), damping_ratio=float(zeta[i]),
                           fill=float(n * vp / np.prod(hi))))
    return scenarios, params


def tile(scenarios, gap=5e-3):
    """One scenario holding every simulation of `scenarios`, each in its own
    region of space, so that one launch per stage of the timestep serves all
    of them.  Simulation i keeps its particles, walls and materials (its
    particle and wall materials become material i of the tiled scenario: the
    per-simulation parameter block), moved by an offset on a square layout in
    x and y whose pitch exceeds any simulation's box plus its walls' extent,
    so that no particle of one simulation comes within reach of another's
    particles or walls.  The shape templates, gravity and time step must be
    shared.  Returns (scenario, layout) with layout holding per simulation
    the particle range, the wall range and the offset."""
    n = len(scenarios)
    if n == 0:
        raise ValueError("no simulations to tile")
    s0 = scenarios[0]
    for sc in scenarios:
        if sc.particle_geometries is not s0.particle_geometries and len(sc.particle_geometries) != len(
                s0.particle_geometries):
            raise ValueError("tiled simulations share their shape templates")
        if not (np.array_equal(sc.gravity, s0.gravity) and sc.dt == s0.dt):
            raise ValueError("tiled simulations share gravity and time step")
        if sc.periodic_x or sc.periodic_y or getattr(sc, "periodic_sector", False) or len(sc.bonds):
            raise ValueError("tiling takes non-periodic simulations without bonds")
        if len(sc.particle_materials) != 1 or len(sc.wall_materials) != 1:
            raise ValueError("each tiled simulation has one particle and one wall material")
    # reach of a simulation around its own domain: its walls' SDF boxes
    reach = []
    for sc in scenarios:
        ext = max([float(np.max(g.size - 1) * g.spacing) for g in sc.wall_geometries], default=0.0)
        reach.append(0.5 * ext)
    span = np.array([sc.domain_max - sc.domain_min for sc in scenarios])
    pitch = float(np.max(span[:, :2].max(axis=1) + 2.0 * np.array(reach))) + gap
    ncol = int(np.ceil(np.sqrt(n)))
    offsets = np.zeros((n, 3))
    for i, sc in enumerate(scenarios):
        offsets[i] = [(i % ncol) * pitch, (i // ncol) * pitch, 0.0] - sc.domain_min
    pos, vel, angvel, quat, mat, geo = [], [], [], [], [], []
    wpos, wvel, wangvel, wquat, wmat, wgeo = [], [], [], [], [], []
    wall_geos, pmat, wmatl, motion = [], [], [], []
    prange, wrange = [], []
    np_, nw_ = 0, 0
    for i, sc in enumerate(scenarios):
        P, W = sc.particles, sc.walls
        pos.append(P.pos + offsets[i]); vel.append(P.vel); angvel.append(P.angvel); quat.append(P.quat)
        mat.append(np.full(len(P), i, np.int32)); geo.append(np.asarray(P.geo, np.int32))
        wpos.append(W.pos + offsets[i]); wvel.append(W.vel); wangvel.append(W.angvel); wquat.append(W.quat)
        wmat.append(np.full(len(W), i, np.int32)); wgeo.append(np.asarray(W.geo, np.int32) + len(wall_geos))
        for (idx, v, w) in sc.wall_motion:
            motion.append((nw_ + idx, v, w))
        wall_geos.extend(sc.wall_geometries)
        pmat.append(sc.particle_materials[0]); wmatl.append(sc.wall_materials[0])
        prange.append((np_, len(P))); wrange.append((nw_, len(W)))
        np_ += len(P); nw_ += len(W)
    lo = np.min([sc.domain_min + offsets[i] for i, sc in enumerate(scenarios)], axis=0)
    hi = np.max([sc.domain_max + offsets[i] for i, sc in enumerate(scenarios)], axis=0)
    cat = np.concatenate
    tiled = S.Scenario(domain_min=lo, domain_max=hi, gravity=s0.gravity, dt=s0.dt, particle_materials=pmat,
                       wall_materials=wmatl, particle_geometries=s0.particle_geometries, wall_geometries=wall_geos,
                       particles=S.Objects(cat(pos), cat(vel), cat(angvel), cat(quat), cat(mat), cat(geo)),
                       walls=S.Objects(cat(wpos), cat(wvel), cat(wangvel), cat(wquat), cat(wmat), cat(wgeo)),
                       wall_motion=motion, name=f"tiled_{n}")
    layout = {"particles": prange, "walls": wrange, "offsets": offsets, "pitch": pitch, "columns": ncol}
    return tiled, layout


class TiledBatch:
    """Independent simulations tiled into one Simulation (see `tile`): every
    kernel of a step runs once for all of them, over the per-simulation
    material blocks and the per-particle wall groups."""

    def __init__(self, scenarios, device=0, precision=0, gap=5e-3):
        self.scenario, self.layout = tile(scenarios, gap=gap)
        self.sim = Simulation.from_scenario(self.scenario, device=device, precision=precision, records=False,
                                            setup=False)
        first = np.concatenate([np.full(n, w0, np.int32) for (_, n), (w0, _) in
                                zip(self.layout["particles"], self.layout["walls"])])
        count = np.concatenate([np.full(n, nw, np.int32) for (_, n), (_, nw) in
                                zip(self.layout["particles"], self.layout["walls"])])
        self.sim.set_wall_groups(first, count)
        self.sim.setup(self.scenario.domain_min, self.scenario.domain_max)
        self.sim.detect()
        self.particles = len(self.scenario.particles)

    def run(self, steps, graph_chunk=0):
        if graph_chunk:
            done = 0
            while done < steps:
                k = min(graph_chunk, steps - done)
                self.sim.step_graph(k)
                done += k
        else:
            self.sim.step(steps)
        self.sim.sync()

    def states(self):
        """Per simulation, its state in its own coordinates."""
        st = self.sim.state()
        out = []
        for i, (p0, n) in enumerate(self.layout["particles"]):
            d = {k: v[p0:p0 + n].copy() for k, v in st.items()}
            d["pos"] -= self.layout["offsets"][i]
            out.append(d)
        return out

    def sync(self):
        self.sim.sync()

    def close(self):
        self.sim.close()


class Batch:
    """Independent simulations, one CUDA stream each."""

    def __init__(self, scenarios, device=0):
        import torch
        self.streams = [torch.cuda.Stream(device=device) for _ in scenarios]
        self.sims = []
        try:
            for sc, st in zip(scenarios, self.streams):
                s = Simulation.from_scenario(sc, device=device, records=False, stream=st.cuda_stream)
                self.sims.append(s)
                s.detect()
        except BaseException:
            # release what was built before the failure
            self.close()
            raise
        self.particles = sum(s.num(False) for s in self.sims)

    def run_graphs(self, steps, chunk):
        """`steps` steps of every simulation, interleaved chunk by chunk."""
        done = 0
        while done < steps:
            k = min(chunk, steps - done)
            for s in self.sims:
                s.step_graph(k)
            done += k
        self.sync()

    def run_sequential(self, steps):
        """The same steps, one simulation after another (each with plain
        launches)."""
        for s in self.sims:
            s.step(steps)
            s.sync()

    def sync(self):
        for s in self.sims:
            s.sync()

    def close(self):
        for s in self.sims:
            s.close()
        self.sims = []


def autotune_chunk(batch, candidates=(25, 50, 100, 200), probe_steps=200):
    """Time `probe_steps` steps of the batch for each candidate chunk length
    (the first chunk of each records its graph) and return the fastest with
    all timings.  Advances the batch by len(candidates) * probe_steps steps."""
    times = {}
    for c in candidates:
        batch.sync()
        t0 = time.perf_counter()
        batch.run_graphs(probe_steps, c)
        times[c] = time.perf_counter() - t0
    best = min(times, key=times.get)
    return best, times


def shard(costs, world):
    """Indices of the simulations each of `world` ranks runs: whole
    simulations, the costliest first, each to the rank with the least work
    so far (ties to the lowest rank).  Deterministic, so every rank computes
    the same split."""
    costs = np.asarray(costs, float)
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += costs[i]
    return [sorted(p) for p in parts]


def run_sharded(scenarios, steps, chunk, rank, world, dist=None, device=0, summary=None, batch_cls=None):
    """Run `steps` steps of this rank's share of `scenarios` (cost: particles
    x steps) as one Batch in graph chunks of `chunk` steps, and return
    {simulation index: summary(simulation)} for every simulation, gathered
    from all ranks (torch.distributed all_gather_object when `dist` is given
    and world > 1).  The default summary is the final mean particle height."""
    batch_cls = Batch if batch_cls is None else batch_cls
    if summary is None:
        def summary(sim):
            return float(sim.state()["pos"][:, 2].mean())
    mine = shard([len(sc.particles) * steps for sc in scenarios], world)[rank]
    local = {}
    error = None
    try:
        if mine:
            b = batch_cls([scenarios[i] for i in mine], device=device)
            try:
                b.run_graphs(steps, chunk)
                for i, sim in zip(mine, b.sims):
                    local[i] = summary(sim)
            finally:
                b.close()
    except Exception as exc:
        if dist is None or world == 1:
            raise
        # every rank still takes part in the gather, then all raise together
        error = f"rank {rank}: {type(exc).__name__}: {exc}"
    if dist is None or world == 1:
        return local
    parts = [None] * world
    dist.all_gather_object(parts, {"error": error, "results": local})
    errors = [p["error"] for p in parts if p["error"]]
    if errors:
        raise RuntimeError("sharded run failed: " + "; ".join(errors))
    out = {}
    for p in parts:
        out.update(p["results"])
    return out


def run_sharded_tiled(scenarios, steps, rank, world, dist=None, device=0, warmup=0, timer=None, tiled_cls=None):
    """This rank's share of `scenarios` (shard, by particles x steps) tiled
    into one simulation (TiledBatch: one launch per stage for the whole
    share): `warmup` untimed steps, then `steps` steps bracketed by
    timer() calls when a timer is given (a callable returning a stop
    callable that returns seconds).  The ranks exchange nothing while they
    run; at the end the final mean particle height of every simulation and
    each rank's seconds are gathered (all_gather_object).  Returns
    ({simulation index: mean height}, [seconds per rank], [indices per
    rank]).  A rank whose share fails still joins the gather, and every rank
    then raises."""
    tiled_cls = TiledBatch if tiled_cls is None else tiled_cls
    parts = shard([len(sc.particles) * steps for sc in scenarios], world)
    mine = parts[rank]
    local, secs, error = {}, 0.0, None
    try:
        if mine:
            tb = tiled_cls([scenarios[i] for i in mine], device=device)
            try:
                if warmup:
                    tb.run(warmup)
                stop = timer() if timer else None
                tb.run(steps)
                secs = stop() if stop else 0.0
                for i, st in zip(mine, tb.states()):
                    local[i] = float(st["pos"][:, 2].mean())
            finally:
                tb.close()
    except Exception as exc:
        if dist is None or world == 1:
            raise
        error = f"rank {rank}: {type(exc).__name__}: {exc}"
    if dist is None or world == 1:
        return local, [secs], parts
    got = [None] * world
    dist.all_gather_object(got, {"error": error, "results": local, "seconds": secs})
    errors = [g["error"] for g in got if g["error"]]
    if errors:
        raise RuntimeError("sharded run failed: " + "; ".join(errors))
    out = {}
    for g in got:
        out.update(g["results"])
    return out, [g["seconds"] for g in got], parts
