"""Autotuners for run parameters that change speed but not results.

`checkpoint_interval` picks the adjoint's checkpoint interval K: every K
steps the forward run keeps a host checkpoint, and the backward pass re-runs
each K-step segment once with recording before sweeping it in reverse.  A
small K costs more checkpoints; a large K records longer segments (device
memory grows with K).  The gradients are the same for every K, because each
re-run repeats the forward run bit for bit.

`launch_shape` picks the narrow phase's grids (blocks per SM of the
selection, the predicate pass, the contact-law pass and the pair sums): the
kernels loop over their work grid-stride, so the shape changes only speed.

`autotune_chunk` in fundem_b200.batch does the same for the number of steps
per CUDA graph in batched runs.
"""
from __future__ import annotations

import time

import numpy as np


def checkpoint_interval(make_sim, steps, dl_dpos, dl_dvel, candidates=(25, 50, 100, 250, 500), max_interval=None):
    """Time forward + backward over `steps` steps for each candidate interval
    and return (best K, {K: seconds}).

    make_sim() returns a fresh Simulation at the initial state, detected.
    Candidates above `steps` or `max_interval` (a memory bound set by the
    caller) are skipped."""
    times = {}
    for k in candidates:
        if k > steps or (max_interval is not None and k > max_interval):
            continue
        sim = make_sim()
        sim.sync()
        t0 = time.perf_counter()
        sim.adjoint_begin(k)
        sim.adjoint_forward(steps)
        sim.adjoint_backward(np.asarray(dl_dpos), np.asarray(dl_dvel))
        sim.sync()
        times[k] = time.perf_counter() - t0
        sim.adjoint_end()
        sim.close()
    if not times:
        raise ValueError("no candidate checkpoint interval fits the run")
    return min(times, key=times.get), times


LAUNCH_SHAPES = ((0, 0, 0, 0), (8, 4, 4, 4), (4, 8, 4, 4), (4, 4, 8, 8), (4, 2, 2, 2), (8, 8, 8, 8), (2, 4, 4, 4))


def launch_shape(sim, steps=20, candidates=LAUNCH_SHAPES, timer=None, restart=False):
    """Time `steps` steps of `sim` under each candidate launch shape
    (select, probe, contact, sums blocks per SM; 0 = default), leave the
    fastest set and return (best, {shape: seconds}).  timer() returns a stop
    callable giving seconds (default: wall clock around synchronised runs).

    restart=False: the candidates run one after another from the current
    state, each after one untimed step; the simulation advances by
    len(candidates) * (steps + 1) steps.  restart=True: every candidate runs
    from the same checkpoint of the current state (written to a temporary
    file), which starts it with a pair-cache rebuild, so that all of them do
    the same work, rebuild steps included (the selection's shape matters only
    there); the simulation ends `steps` steps after the checkpoint."""
    times = {}
    tmp = None
    if restart:
        import os
        import tempfile
        fd, tmp = tempfile.mkstemp(suffix=".fdck")
        os.close(fd)
        sim.checkpoint_write(tmp)
    try:
        for shape in candidates:
            if restart:
                sim.checkpoint_read(tmp)
            sim.set_launch_shape(*shape)
            if not restart:
                sim.step(1)
            sim.sync()
            if timer is None:
                t0 = time.perf_counter()
                sim.step(steps)
                sim.sync()
                times[tuple(shape)] = time.perf_counter() - t0
            else:
                stop = timer()
                sim.step(steps)
                times[tuple(shape)] = stop()
                sim.sync()
    finally:
        if tmp is not None:
            import os
            os.remove(tmp)
    best = min(times, key=times.get)
    sim.set_launch_shape(*best)
    return best, times
