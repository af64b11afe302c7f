"""Autotuners for run parameters that change speed but not results.

`checkpoint_interval` picks the adjoint's checkpoint interval K: every K
steps the forward run keeps a host checkpoint, and the backward pass re-runs
each K-step segment once with recording before sweeping it in reverse.  A
small K costs more checkpoints; a large K records longer segments (device
memory grows with K).  The gradients are the same for every K, because each
re-run repeats the forward run bit for bit.

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
