#!/usr/bin/env python
"""Throughput of the level-set DEM timestep on B200: particle-steps/s.

    python bench.py [--gpus N --steps K --warmup W] [--impl fundem|reference]

Workload (default): the scaled, periodic, bonded column -- 262,144
superellipsoids from 8 templates (32^3 SDFs, 642 surface nodes), periodic in
x and y, floor wall and a top platen that starts on the bed and moves down
at 1 m/s, V-model bonds between pairs whose surface gap is below 0.05 of the
mean diameter, dt = 5e-7 s, FP64.  A step is one pass of the whole timestep
(kicks, drift, hashing, broad phase, narrow phase + contact law, ghosts,
bonds, reduction) over the resident state.  The default warm-up (1000 steps)
puts the timed window in the compression phase.  Inputs are larger than L2
(state + templates + lists are several hundred MB), so no L2 flush is needed
between steps.

The `mixed` object compares the mixed-precision mode with FP64 on the same
workload: two fresh simulations run --error-steps steps, their positions are
compared, then each runs K timed steps from there.

--impl reference times the CPU restatement of the reference algorithm (the
reference itself has no CPU code) on a bounded sample of the same workload,
with all host threads.

Under torchrun each rank runs an independent replica (the path does not
shard: a single simulation lives on one GPU); value = all ranks' particle
steps / the slowest rank's time.
"""
from __future__ import annotations

import argparse
import faulthandler
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s"
PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
# algorithmic bytes per unit (FP64): per particle-step and per node-contact-step
BYTES_PARTICLE_STEP = 216
BYTES_CONTACT_STEP = 64
BYTES_BOND_STEP = 340


def log(*a):
    print(*a, file=sys.stderr, flush=True)


class ClockSampler:
    """SM clock, power and clock-event reasons sampled during the timed
    region: NVML in a thread every 5 ms (the region can be a few tens of
    milliseconds), or nvidia-smi every 200 ms where NVML is missing."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clock-event reason bits
    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown"}

    def __init__(self, index, period_s=0.005):
        self.index = index
        self.period = period_s
        self.samples = []   # (sm_mhz, max_mhz, power_w, reason bits)
        self.proc = None
        self.nvml = None
        self._stop = threading.Event()

    def _nvml_handle(self):
        """The NVML handle of CUDA device `index`, matched by UUID (NVML and
        CUDA may number devices differently), else by index."""
        import pynvml
        pynvml.nvmlInit()
        want = None
        try:
            import torch
            want = str(torch.cuda.get_device_properties(self.index).uuid).lower()
        except Exception:
            pass
        if want:
            for i in range(pynvml.nvmlDeviceGetCount()):
                h = pynvml.nvmlDeviceGetHandleByIndex(i)
                u = pynvml.nvmlDeviceGetUUID(h)
                u = (u.decode() if isinstance(u, bytes) else str(u)).lower()
                if u.endswith(want):
                    return pynvml, h
        return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def start(self):
        try:
            self.nvml, h = self._nvml_handle()
            self.thread = threading.Thread(target=self._poll_nvml, args=(h,), daemon=True)
            self.thread.start()
            return
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read_smi, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _poll_nvml(self, h):
        N = self.nvml
        mx = N.nvmlDeviceGetMaxClockInfo(h, N.NVML_CLOCK_SM)
        get_reasons = getattr(N, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            N.nvmlDeviceGetCurrentClocksThrottleReasons
        while not self._stop.is_set():
            try:
                self.samples.append((float(N.nvmlDeviceGetClockInfo(h, N.NVML_CLOCK_SM)), float(mx),
                                     N.nvmlDeviceGetPowerUsage(h) / 1e3, int(get_reasons(h))))
            except Exception:
                pass
            time.sleep(self.period)

    def _read_smi(self):
        names = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20, "sw_power_cap": 0x4}
        for line in self.proc.stdout:
            s = [x.strip() for x in line.split(",")]
            if len(s) < 9 or not s[1].replace(".", "").isdigit():
                continue
            bits = 0
            for k, nm in enumerate(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")):
                if "Active" in s[5 + k] and "Not" not in s[5 + k]:
                    bits |= names[nm]
            pw = float(s[3]) if s[3].replace(".", "").isdigit() else float("nan")
            self.samples.append((float(s[1]), float(s[2]), pw, bits))

    def stop(self):
        self._stop.set()
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if getattr(self, "thread", None):
            self.thread.join(timeout=5)
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0,
                    "source": "nvml" if self.nvml else ("nvidia-smi" if self.proc else "unavailable")}
        sm = [x[0] for x in self.samples]
        reasons = set()
        for x in self.samples:
            for bit, nm in self.REASONS.items():
                if x[3] & bit:
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)), "sm_min_mhz": float(min(sm)), "sm_max_mhz": max(x[1] for x in self.samples),
                "power_w_max": float(np.nanmax([x[2] for x in self.samples])), "reasons": sorted(reasons),
                "samples": len(self.samples), "source": "nvml" if self.nvml else "nvidia-smi"}


def pinned_like(a):
    """A copy of a numpy array in page-locked host memory."""
    import torch
    t = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
    out = t.numpy()  # shares the tensor's memory and keeps the tensor alive
    out[...] = a
    return out


def peaks():
    try:
        with open(PEAKS) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# CPU baseline: the oracle (a restatement of the reference algorithm) on a
# bounded sample of the same workload, all host threads
# ---------------------------------------------------------------------------
def cpu_sample_scenario(n=2048):
    from fundem_b200 import scenario as S
    rng = np.random.default_rng(7)
    geos = S.superellipsoid_templates(rng, 8, n=32, level=3, density=2500.0, explicit_mass=True)
    rb = max(S.node_radius(g) for g in geos)
    sc = S.bonded_periodic(n=n, n_templates=8, seed=7, pitch=2.0 * rb * 1.01, resolve=False, dt=5e-7)
    return sc


def cpu_baseline(seconds=15.0, n=2048):
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    O.set_threads(threads)
    sc = cpu_sample_scenario(n)
    w = O.OracleWorld.from_scenario(sc)
    w.initial_detect()
    w.step(1)
    steps, t0 = 0, time.perf_counter()
    while time.perf_counter() - t0 < seconds:
        w.step(1)
        steps += 1
    dt = time.perf_counter() - t0
    return {"value": n * steps / dt, "unit": METRIC, "cores": threads, "kind": "port",
            "sample": f"{n} particles of the bonded periodic column (8 templates, 32^3 SDF, 642 nodes, "
                      f"{len(sc.bonds)} bonds), {steps} steps in {dt:.1f} s"}


# ---------------------------------------------------------------------------
def run_reference(args, rank, world):
    if rank != 0:
        return
    res = cpu_baseline(seconds=max(5.0, 3.0 * args.steps / 10.0), n=args.cpu_sample)
    line = {"metric": METRIC, "value": res["value"], "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": "bonded periodic column, bounded CPU sample", "sample_particles": args.cpu_sample},
            "cpu_baseline": res,
            "e2e": {"value": res["value"], "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_fundem(args, rank, world, dist):
    import torch
    import fundem_b200 as F
    from fundem_b200 import build, workloads

    build.build()
    dev = int(os.environ.get("LOCAL_RANK", 0))

    def log0(*a):
        if rank == 0:
            log(*a)
    torch.cuda.set_device(dev)
    t_build = time.perf_counter()
    sim, sc, info = workloads.bonded_column(n=args.n, footprint=tuple(args.footprint), seed=1 + rank, device=dev,
                                            settle_steps=args.settle_steps, log=log if rank == 0 else None)
    t_build = time.perf_counter() - t_build
    n = info["n"]
    g = np.asarray(sc.gravity, float)
    dt = sc.dt
    log0(f"workload built in {t_build:.1f} s; {args.warmup} warm-up steps")
    sim.set_pair_cache(args.pair_cache, args.pair_skin)
    sim.step(args.warmup)
    sim.sync()
    shape = None
    if not args.no_autotune:
        # the narrow phase's launch shape, tuned on this state (untimed;
        # results do not depend on it)
        from fundem_b200 import autotune
        tune_steps = 40
        best, times = autotune.launch_shape(sim, steps=tune_steps, restart=True)
        shape = {"chosen_blocks_per_sm": list(sim.launch_shape()),
                 "order": ["select", "probe", "contact", "sums"],
                 "ms_per_step": {",".join(str(v) for v in k): 1e3 * t / tune_steps for k, t in times.items()},
                 "note": f"autotune.launch_shape after the warm-up steps: every candidate runs {tune_steps} steps "
                         "from one checkpoint of that state (a pair-cache rebuild first, then the same steps "
                         "for all), 0 = default"}
        log0(f"launch shape {sim.launch_shape()}")
    if not args.no_graph:
        # the headline replays one CUDA graph of K steps (fundem_step_graph);
        # record it here, untimed, for both list generations it can start on
        sim.step_graph(args.steps)
        sim.step_graph(args.steps)
        sim.sync()
    pc0 = sim.pair_cache_stats()
    pairs = sim.num_pairs(0)
    contacts = sim.num_contacts(0) + sim.num_contacts(1) + sum(sim.num_contacts(k) for k in (2, 3, 4))
    nbonds = int(sim.bonds()["activated"].sum())
    l0 = sim.launch_count()
    clocks = ClockSampler(dev)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    time.sleep(0.02)  # the sampler's first reading precedes the region
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if args.profile:
        torch.cuda.profiler.start()
    # the headline: K steps, no kernel timers (one graph replay, or plain
    # launches with --no-graph)
    e0.record()
    if args.no_graph:
        sim.step(args.steps)
    else:
        sim.step_graph(args.steps)
    e1.record()
    torch.cuda.synchronize()
    if args.profile:
        torch.cuda.profiler.stop()
    clk = clocks.stop()
    sim.sync()
    if dist:
        dist.barrier()
    ms = e0.elapsed_time(e1)
    launches = sim.launch_count() - l0
    pc1 = sim.pair_cache_stats()
    contacts_end = sim.num_contacts(0) + sim.num_contacts(1) + sum(sim.num_contacts(k) for k in (2, 3, 4))
    t_max, value = aggregate(ms, n, args.steps, world, dist, "cuda")
    log0(f"timed: {ms / args.steps:.4f} ms/step, clocks {clk}")
    # the same K steps with plain launches (every kernel launched from the
    # host), for comparison
    torch.cuda.synchronize()
    e0.record()
    sim.step(args.steps)
    e1.record()
    torch.cuda.synchronize()
    plain_ms = e0.elapsed_time(e1) / args.steps
    log0(f"plain launches: {plain_ms:.4f} ms/step")
    # the same K steps again with the kernel-group timers on (CUDA events on
    # the simulation's stream around each group): per-kernel times and the
    # roofline's launch duration
    sim.set_profiling(True)
    sim.kernel_times()
    sim.step(args.steps)
    sim.sync()
    kt = sim.kernel_times()
    sim.set_profiling(False)

    # end to end through the C ABI with host buffers in pinned memory: upload
    # the state, run the steps reading back the status word every step,
    # download the state
    st = sim.state()
    host = {k: pinned_like(v) for k, v in st.items()}
    back = {k: pinned_like(v) for k, v in st.items()}
    state_bytes = sum(v.nbytes for v in host.values())
    e2e_steps = 0 if args.no_e2e else args.steps
    if e2e_steps:
        # each step replays a one-step CUDA graph (fundem_step_graph);
        # record it once, outside the timing
        sim.step_graph(1)
        sim.sync()
    # every step's status word goes to a page-locked ring, read after the sync
    ring = torch.zeros(max(e2e_steps, 1), dtype=torch.int32, pin_memory=True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    sim.set_state(**host)
    for k in range(e2e_steps):
        sim.step_graph(1)
        sim.status_word_to(ring.data_ptr() + 4 * k)
    sim.state(out=back)
    sim.sync()
    t_e2e = time.perf_counter() - t0
    status_ok = bool(torch.all(ring[:e2e_steps] == 0).item()) if e2e_steps else None
    log0(f"end to end: {t_e2e:.4f} s, status words clean: {status_ok}")
    # narrow-phase work counters, on a few extra steps outside the timed regions
    wc_steps = 10
    sim.set_profiling(False, counters=True)
    sim.work_counters()
    sim.step(wc_steps)
    wc = sim.work_counters()
    sim.set_profiling(False)
    e2e_val = 0.0
    if e2e_steps:
        _, e2e_val = aggregate(1e3 * t_e2e, n, e2e_steps, world, dist, "cuda")
    # resident state, steps replayed from CUDA graphs of GRAPH_CHUNK steps
    graph = None
    if args.steps >= GRAPH_CHUNK:
        sim.step_graph(GRAPH_CHUNK)
        sim.sync()
        torch.cuda.synchronize()
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        chunks = args.steps // GRAPH_CHUNK
        g0.record()
        for _ in range(chunks):
            sim.step_graph(GRAPH_CHUNK)
        g1.record()
        torch.cuda.synchronize()
        sim.sync()
        g_max, g_val = aggregate(g0.elapsed_time(g1), n, chunks * GRAPH_CHUNK, world, dist, "cuda")
        graph = {"value": g_val, "unit": METRIC, "ms_per_step": g_max / (chunks * GRAPH_CHUNK),
                 "chunk": GRAPH_CHUNK, "note": "resident state; fundem_step_graph replays, no kernel timers"}

    # mixed precision against FP64 on the same workload: two fresh simulations
    # from the initial state, `error_steps` steps each, positions compared
    # (minimum image across the periodic seams), then K timed steps each
    mixed = None if args.no_mixed else mixed_vs_fp64(sc, dev, args, dist, world)
    batched = None
    if not args.no_batch and world > 1:
        # every rank takes part (the sweep is split across them)
        try:
            batched = batched_sharded(args, rank, world, dist, dev)
        except Exception as exc:  # an auxiliary figure: report, do not fail the run
            batched = {"error": f"{type(exc).__name__}: {exc}"}
    elif not args.no_batch and rank == 0:
        try:
            batched = batched_cost(args, dev)
        except Exception as exc:  # an auxiliary figure: report, do not fail the run
            batched = {"error": f"{type(exc).__name__}: {exc}"}
    adjoint = None
    if not args.no_adjoint and rank == 0:
        try:
            adjoint = adjoint_cost(args, dev)
        except Exception as exc:  # an auxiliary figure: report, do not fail the run
            adjoint = {"error": f"{type(exc).__name__}: {exc}"}

    ref_gpu = None
    if rank == 0 and world == 1 and not args.no_reference_gpu:
        try:
            ref_gpu = reference_gpu_time(sc, args)
        except Exception as exc:  # an auxiliary figure: report, do not fail the run
            ref_gpu = {"error": f"{type(exc).__name__}: {exc}"}
    if rank != 0:
        return
    pk, pk_kind = peaks()
    nar_ms, nar_n = kt["narrow_pp"]
    nar_avg = nar_ms / max(nar_n, 1)
    # algorithmic bytes of one particle-particle narrow-phase launch: every
    # particle's state (216 B) plus every node contact's history and ids (64 B)
    nar_bytes = BYTES_PARTICLE_STEP * n + BYTES_CONTACT_STEP * 0.5 * (contacts + contacts_end)
    achieved = nar_bytes / (nar_avg / 1e3) / 1e9 if nar_avg > 0 else None
    step_bytes = BYTES_PARTICLE_STEP * n + BYTES_CONTACT_STEP * 0.5 * (contacts + contacts_end) + BYTES_BOND_STEP * nbonds
    traffic_per_pair = profiled_traffic_per_pair()
    cpu = None
    if world == 1 and not args.no_cpu:
        cpu = cpu_baseline(seconds=args.cpu_seconds, n=args.cpu_sample)
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "bonded periodic column (config 1 shape)", "particles_per_gpu": n,
                   "templates": 8, "sdf_grid": "32^3", "surface_nodes": 642, "dt": dt,
                   "bonds": info["bonds"], "periodic": "xy", "precision": "fp64",
                   "footprint": info["footprint"], "layers": info["layers"],
                   "l2": "inputs larger than L2 (no flush)", "parallelism": f"replicas x{world}",
                   "pairs": pairs, "node_contacts": contacts, "node_contacts_end": contacts_end,
                   "active_bonds": nbonds, "setup_s": round(t_build, 1),
                   "settle": {"steps": info["settle_steps"], "dt": info["settle_dt"],
                              "peak_speed_m_s": info["settle_peak_speed"], "settled": info["settled"],
                              "kinetic_energy_j": info["settle_kinetic_energy"],
                              "kinetic_energy_peak_j": info["settle_kinetic_energy_peak"],
                              "coordination": info["coordination"],
                              "node_contacts": info["settled_node_contacts"]},
                   "timed_from": "the settled, bonded bed with the platen released (workloads.bonded_column)"},
        "e2e": {"value": e2e_val, "unit": METRIC, "h2d_bytes_per_step": state_bytes / args.steps,
                "d2h_bytes_per_step": 4 + state_bytes / args.steps,
                "status_words_clean": status_ok,
                "note": "state uploaded from page-locked host arrays, each step a one-step CUDA-graph replay "
                        "(fundem_step_graph) followed by a copy of its status word into a page-locked ring "
                        "(checked after the final sync), state downloaded"},
        "graph": graph,
        "headline_path": "plain launches (fundem_step)" if args.no_graph else
                         "one CUDA graph of K steps replayed (fundem_step_graph), recorded before the timed region",
        "plain_launches_ms_per_step": plain_ms,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": pk, "unit": "GB/s",
                     "frac": (achieved / pk) if achieved else None,
                     "traffic": (traffic_per_pair * pairs) if traffic_per_pair else None,
                     "traffic_source": TRAFFIC_PROFILE + " (ncu DRAM bytes per candidate pair x pairs)"
                     if traffic_per_pair else None,
                     "kernel": "k_narrow<PP> (narrow phase + contact law)", "peak_source": pk_kind,
                     "kernel_ms": nar_avg, "algorithmic_bytes": nar_bytes,
                     "step_achieved_gbs": step_bytes / (t_max / args.steps / 1e3) / 1e9},
        "roofline_fp64": fp64_roofline(wc, wc_steps, nar_avg),
        "contact_updates_per_s": world * 0.5 * (contacts + contacts_end) * args.steps / (t_max / 1e3),
        "pair_cache": {"skin_m": pc1[2], "rebuilds_in_timed_steps": pc1[0] - pc0[0],
                       "timed_steps": pc1[1] - pc0[1],
                       "note": "candidate pairs and contact slots of the particle-particle, particle-wall and "
                               "image lists kept between rebuilds (a particle drifting half the skin rebuilds "
                               "them); on the steps between, the exact FP64 node predicate runs on every slot "
                               "that a per-pair bound on the SDF's change since the rebuild does not rule out"},
        "kernel_ms_per_step": {k: v[0] / max(args.steps, 1) for k, v in kt.items()},
        "launch_shape": shape,
        "kernel_timing": "a second pass of K steps right after the headline, with CUDA-event timers on the "
                         "simulation's stream around each kernel group (all stages on that one stream)",
        "streams": "headline and plain launches: the particle-particle list on the simulation's stream; the "
                   "particle-wall list and the image lists (with the bonds at the end of one of them) on two "
                   "more streams, forked after the hash stage and joined before the force sums",
        "reference_gpu": ref_gpu,
        "narrow_work_per_step": {"pairs": wc[0] / wc_steps, "clusters": wc[1] / wc_steps,
                                 "clusters_kept": wc[2] / wc_steps, "node_contacts": wc[3] / wc_steps,
                                 "exact_node_tests": wc[4] / wc_steps,
                                 "cached_slots_tested": wc[5] / wc_steps,
                                 "cached_slots_skipped_by_bound": wc[6] / wc_steps},
        "mixed": mixed,
        "adjoint": adjoint,
        "batched": batched,
        "cpu_baseline": cpu,
        "clocks": clk,
        "gpu_launches": launches,
    }
    print(json.dumps(line), flush=True)


GRAPH_CHUNK = 50  # steps per CUDA graph in the graph-replay measurement
# ncu summary holding the narrow phase's DRAM bytes per candidate pair
TRAFFIC_PROFILE = "profiles/narrow_pp_traffic_bonded_column_65k.md"


# the secondary flop model of the narrow phase: about 100 FP64 flops per node
# given the exact predicate (two rotations, the grid mapping, the trilinear
# value) and about 120 per contact (normal, contact point, the contact law)
FLOPS_PER_TESTED_NODE = 100.0
FLOPS_PER_CONTACT = 120.0
FP64_PEAK_TFLOPS = 37.0  # nominal B200 FP64 (datasheet); no measured figure exists


def fp64_roofline(wc, wc_steps, narrow_ms):
    """The particle-particle narrow phase against FP64 throughput: flops per
    step from the flop model and the work counters (nodes given the exact
    predicate by the cached predicate pass, node contacts), over the group's
    time per step."""
    if not narrow_ms or wc_steps <= 0:
        return None
    tested = wc[5] / wc_steps if len(wc) > 5 else 0.0
    contacts = wc[3] / wc_steps
    flops = FLOPS_PER_TESTED_NODE * tested + FLOPS_PER_CONTACT * contacts
    achieved = flops / (narrow_ms / 1e3) / 1e12
    return {"bound": "fp64", "achieved": achieved, "peak": FP64_PEAK_TFLOPS, "unit": "TFLOP/s",
            "frac": achieved / FP64_PEAK_TFLOPS, "peak_source": "nominal (no measured FP64 figure)",
            "flops_per_step": flops, "model": f"{FLOPS_PER_TESTED_NODE:g} per node tested, "
                                              f"{FLOPS_PER_CONTACT:g} per contact"}


def profiled_traffic_per_pair():
    """DRAM bytes per candidate pair of the particle-particle narrow phase,
    from the committed ncu summary (None when it is absent)."""
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), TRAFFIC_PROFILE)
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_pair"):
                    return float(line.split("=")[1])
    except OSError:
        pass
    return None


def reference_gpu_time(sc, args):
    """The reference's own CUDA build (oracle/_ref/ref_driver: its LSSolver and
    kernels compiled from its sources, no change) on the same settled state,
    same B200: wall time between the solver hooks of two steps, after a
    device synchronisation at each end, with no output frame between them
    (the reference writes frames at the start and end of a solve).  The
    reference starts without the tangential-spring history of the settle."""
    import shutil
    import tempfile
    from oracle import scenario_io
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_driver")
    if not os.path.exists(exe):
        return {"unavailable": "oracle/_ref/ref_driver not built (needs the reference sources)"}
    steps_ref, lo = args.reference_gpu_steps, 10
    out = tempfile.mkdtemp(prefix="fundem_ref_")
    try:
        path = os.path.join(out, "scenario.bin")
        scenario_io.write_reference_scenario(sc, path, steps_ref)
        t0 = time.time()
        r = subprocess.run([exe, path, out, "timing", str(lo), str(steps_ref - 5), "exit"], capture_output=True,
                           text=True, timeout=args.reference_gpu_timeout)
        wall = time.time() - t0
        if r.returncode != 0:
            return {"error": f"ref_driver exit {r.returncode}: {r.stderr[-300:]}"}
        meta = {}
        with open(os.path.join(out, "meta.txt")) as f:
            for line in f:
                k, v = line.split(None, 1)
                meta[k] = v.strip()
    finally:
        shutil.rmtree(out, ignore_errors=True)
    ms = 1e3 * float(meta["window_seconds"]) / float(meta["window_steps"])
    n = len(sc.particles)
    return {"ms_per_step": ms, "value": n / (ms / 1e3), "unit": METRIC, "window_steps": [lo, steps_ref - 5],
            "wall_s": round(wall, 1), "what": "the reference's CUDA build, same scenario and state, same GPU"}


def aggregate(ms, n, steps, world, dist, device):
    """Whole-job throughput of `world` replicas of n particles each: the
    slowest rank's time (a MAX all-reduce, every rank takes part) and
    world * n * steps / that time, in particle-steps/s."""
    t_max = ms
    if dist:
        import torch
        t = torch.tensor([float(ms)], device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_max = float(t.item())
    return t_max, world * n * steps / (t_max / 1e3)


def mixed_vs_fp64(sc, dev, args, dist, world):
    import torch
    import fundem_b200 as F
    n = len(sc.particles)
    sims = {}
    for prec in (F.FP64, F.FP32_MIXED):
        s = F.Simulation.from_scenario(sc, device=dev, precision=prec, records=False)
        s.detect()
        s.step(args.error_steps)
        s.sync()
        sims[prec] = s
    a, b = sims[F.FP64].state(), sims[F.FP32_MIXED].state()
    L = np.array([sc.domain_max[0] - sc.domain_min[0], sc.domain_max[1] - sc.domain_min[1]])
    d = a["pos"] - b["pos"]
    for k in range(2):
        if (sc.periodic_x, sc.periodic_y)[k]:
            d[:, k] -= L[k] * np.round(d[:, k] / L[k])
    dx = np.linalg.norm(d, axis=1)
    rel = dx / np.maximum(np.linalg.norm(a["pos"], axis=1), 1e-300)
    norm_rel = float(np.linalg.norm(d) / np.linalg.norm(a["pos"]))
    dq = 1.0 - np.abs(np.sum(a["quat"] * b["quat"], axis=1))
    ms = {}
    for prec, s in sims.items():
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if not args.no_graph:
            # timed as the headline: a K-step graph, recorded untimed
            s.step_graph(args.steps)
            s.step_graph(args.steps)
            s.sync()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e0.record()
        if args.no_graph:
            s.step(args.steps)
        else:
            s.step_graph(args.steps)
        e1.record()
        torch.cuda.synchronize()
        s.sync()
        t = e0.elapsed_time(e1)
        if dist:
            tt = torch.tensor([t], device="cuda")
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            t = float(tt.item())
        ms[prec] = t / args.steps
    for s in sims.values():
        s.close()
    gate = 1e-5
    return {"value": world * n / (ms[F.FP32_MIXED] / 1e3), "unit": METRIC, "ms_per_step": ms[F.FP32_MIXED],
            "fp64_ms_per_step_same_state": ms[F.FP64], "speedup_vs_fp64": ms[F.FP64] / ms[F.FP32_MIXED],
            "dtype": "f32 contact and bond laws, f64 integration and spring history",
            "timed_after_steps": args.error_steps,
            "error_vs_fp64": {"steps": args.error_steps, "normwise_rel_position": norm_rel,
                              "p99_rel_position": float(np.percentile(rel, 99)), "max_rel_position": float(rel.max()),
                              "max_abs_position_m": float(dx.max()), "p99_abs_position_m": float(np.percentile(dx, 99)),
                              "max_quaternion_error": float(dq.max()), "gate_rel_position": gate,
                              "pass": bool(norm_rel <= gate and np.percentile(rel, 99) <= gate),
                              "gate_metric": "||X_mixed - X_fp64|| / ||X_fp64|| and the 99th percentile of "
                                             "|x_mixed - x_fp64| / |x_fp64| over particles"}}


def adjoint_cost(args, dev):
    """Config 3: the adjoint of the pour (4096 particles, 2 templates, six
    walls, dt = 1e-6 s, args.adjoint_steps steps, a checkpoint every 500)
    against the plain forward run, in FP64 and FP32_MIXED, from the poured
    bed (untimed: the library's own steps at 5e-6 s until the kinetic energy
    falls below 1e-3 of the fall's peak or 40,000 steps).  Loss: the final
    packing fraction, N V / (A H) with A the box's floor area and H twice the
    mean particle height (the height of a bed filled evenly), plus the
    mean-square displacement of 64 tagged particles."""
    import fundem_b200 as F
    from fundem_b200 import workloads
    sim, sc = workloads.adjoint_pour(n=4096, device=dev, settle_steps=40000)
    n = len(sc.particles)
    x0 = np.array(sc.particles.pos, copy=True)
    sim.close()
    masses = np.array([g.mass for g in sc.particle_geometries])[sc.particles.geo]
    vol = float(np.sum(masses) / 2500.0)           # the templates' density
    lo, hi = sc.walls.pos.min(axis=0), sc.walls.pos.max(axis=0)
    area, zfloor = float((hi[0] - lo[0]) * (hi[1] - lo[1])), float(lo[2])
    steps, K = args.adjoint_steps, 500

    def run(precision):
        s = F.Simulation.from_scenario(sc, device=dev, records=False)
        s.set_precision(precision)
        s.detect()
        s.sync()
        t0 = time.perf_counter()
        s.step(steps)
        s.sync()
        t_fwd = time.perf_counter() - t0
        s.close()
        s = F.Simulation.from_scenario(sc, device=dev, records=False)
        s.set_precision(precision)
        s.detect()
        s.adjoint_begin(K)
        t0 = time.perf_counter()
        s.adjoint_forward(steps)
        t_rec = time.perf_counter() - t0
        st = s.state()
        tag = np.arange(0, n, n // 64)[:64]
        H = 2.0 * float(np.mean(st["pos"][:, 2] - zfloor))
        phi = vol / (area * H)
        msd = float(np.mean(np.sum((st["pos"][tag] - x0[tag]) ** 2, axis=1)))
        dl_dx = np.zeros((n, 3))
        dl_dx[:, 2] = -phi / H * 2.0 / n
        dl_dx[tag] += 2.0 * (st["pos"][tag] - x0[tag]) / len(tag)
        contacts = s.num_contacts(F.PP) + s.num_contacts(F.PW)
        t0 = time.perf_counter()
        gv0, gp = s.adjoint_backward(dl_dx, np.zeros((n, 3)))
        t_bwd = time.perf_counter() - t0
        s.adjoint_end()
        s.close()
        return {"node_contacts_at_end": contacts, "loss": phi + msd, "packing_fraction": phi, "tagged_msd_m2": msd,
                "forward_s": t_fwd, "recorded_forward_s": t_rec,
                "backward_s": t_bwd, "backward_over_forward": t_bwd / t_fwd,
                "total_over_forward": (t_rec + t_bwd) / t_fwd, "dl_dparams": gp[0].tolist()}

    out = {"workload": "adjoint pour (config 3): 4096 superellipsoids, 2 templates, six walls, dt 1e-6 s, from "
                       "the poured bed; loss: packing fraction (bed height twice the mean particle height) + "
                       "mean-square displacement of 64 tagged particles",
           "steps": steps, "checkpoint_interval": K, "settle": sc.settle}
    out.update(run(F.FP64))
    out["fp32_mixed"] = run(F.FP32_MIXED)
    out["dl_dparams_order"] = ["kn", "ks", "damping ratio", "mu"]
    out["note"] = ("backward re-runs each checkpoint segment once with recording, then sweeps it in reverse; "
                   "wall-clock times, the calls synchronise; fp32_mixed: the FP32_MIXED step and its adjoint "
                   "(the recorded single-precision run swept with double-precision Jacobians)")
    return out


def batched_cost(args, dev):
    """The calibration sweep: args.batch_sims independent pours of uneven size
    (log-uniform in [500, 20000] particles, per-simulation kn, friction and
    damping), args.batch_steps steps each, run tiled into one simulation (one
    launch per stage of the timestep over all simulations, per-simulation
    material blocks and wall groups) and one at a time; then the adjoint of a
    tiled subset against its forward run."""
    import torch
    import fundem_b200 as F
    from fundem_b200 import batch
    t0 = time.perf_counter()
    scs, params = batch.calibration_scenarios(n_sims=args.batch_sims, seed=1)
    t_build = time.perf_counter() - t0
    t0 = time.perf_counter()
    tb = batch.TiledBatch(scs, device=dev)
    t_setup = time.perf_counter() - t0
    particles = tb.particles
    tb.run(args.batch_warmup)  # untimed: list growth and the first cache builds
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    tb.sim.step(args.batch_steps)
    e1.record()
    torch.cuda.synchronize()
    tb.sync()
    t_tiled = e0.elapsed_time(e1) / 1e3
    launches = tb.sim.launch_count()
    tb.close()
    seq = batch.Batch(scs, device=dev)
    seq.sync()
    seq.run_sequential(args.batch_warmup)  # the same warm-up steps, untimed
    t0 = time.perf_counter()
    seq.run_sequential(args.batch_steps)
    t_seq = time.perf_counter() - t0
    seq.close()
    ps = particles * args.batch_steps
    out = {"workload": "calibration sweep: pours of 500-20,000 particles (log-uniform), kn, friction and damping "
                       "per simulation, the small pour's shapes, fill ratio 0.4, dt 1e-6 s",
           "simulations": len(scs), "particles": particles, "steps": args.batch_steps,
           "warmup_steps": args.batch_warmup,
           "tiled_s": t_tiled, "sequential_s": t_seq, "speedup": t_seq / t_tiled,
           "tiled_particle_steps_per_s": ps / t_tiled, "sequential_particle_steps_per_s": ps / t_seq,
           "scenario_build_s": round(t_build, 1), "tiled_setup_s": round(t_setup, 1),
           "note": "tiled: every simulation in its own region of one Simulation, one launch per stage for all "
                   "(CUDA events); sequential: the same simulations stepped one after another with plain launches "
                   "(wall clock around synchronised runs)"}
    # the adjoint of a tiled subset: per-simulation parameter gradients from one backward sweep
    try:
        sub = scs[: args.batch_adjoint_sims]
        steps, K = args.batch_adjoint_steps, max(args.batch_adjoint_steps // 4, 1)
        t2 = batch.TiledBatch(sub, device=dev)
        n = t2.particles
        t2.sim.sync()
        t0 = time.perf_counter()
        t2.sim.step(steps)
        t2.sim.sync()
        t_fwd = time.perf_counter() - t0
        t2.close()
        t2 = batch.TiledBatch(sub, device=dev)
        t2.sim.adjoint_begin(K)
        t0 = time.perf_counter()
        t2.sim.adjoint_forward(steps)
        t_rec = time.perf_counter() - t0
        dl_dx = np.zeros((n, 3))
        dl_dx[:, 2] = 1.0 / n            # loss: mean particle height of every simulation together
        t0 = time.perf_counter()
        gv0, gp = t2.sim.adjoint_backward(dl_dx, np.zeros((n, 3)))
        t_bwd = time.perf_counter() - t0
        t2.sim.adjoint_end()
        t2.close()
        out["adjoint"] = {"simulations": len(sub), "particles": n, "steps": steps, "checkpoint_interval": K,
                          "forward_s": t_fwd, "recorded_forward_s": t_rec, "backward_s": t_bwd,
                          "total_over_forward": (t_rec + t_bwd) / t_fwd,
                          "dl_dkn_first_sims": [float(g[0]) for g in gp[:4]]}
    except Exception as exc:  # an auxiliary figure: report, do not fail the run
        out["adjoint"] = {"error": f"{type(exc).__name__}: {exc}"}
    return out


def batched_sharded(args, rank, world, dist, dev):
    """The calibration sweep split across the ranks: whole simulations per
    GPU, the costliest first (batch.shard by particles x steps); each rank
    tiles its share into one simulation and runs args.batch_warmup untimed
    and args.batch_steps timed steps.  The ranks exchange nothing while they
    run; the results and each rank's device time (CUDA events) are gathered
    at the end, and the job's time is the slowest rank's."""
    import torch
    from fundem_b200 import batch
    scs, _ = batch.calibration_scenarios(n_sims=args.batch_sims, seed=1)

    def timer():
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()

        def stop():
            e1.record()
            torch.cuda.synchronize()
            return e0.elapsed_time(e1) / 1e3
        return stop
    res, secs, parts = batch.run_sharded_tiled(scs, args.batch_steps, rank, world, dist=dist, device=dev,
                                               warmup=args.batch_warmup, timer=timer)
    total = sum(len(sc.particles) for sc in scs)
    t = max(secs)
    return {"workload": "calibration sweep split across GPUs: whole simulations per rank, largest first, each "
                        "rank's share tiled into one simulation",
            "simulations": len(scs), "particles": total, "steps": args.batch_steps,
            "warmup_steps": args.batch_warmup, "ranks": world,
            "simulations_per_rank": [len(p) for p in parts],
            "particles_per_rank": [int(sum(len(scs[i].particles) for i in p)) for p in parts],
            "seconds_per_rank": secs, "job_s": t, "particle_steps_per_s": total * args.batch_steps / t,
            "results_gathered": len(res),
            "note": "strong scaling of a fixed sweep; no exchange while running (the per-simulation results "
                    "are gathered once at the end)"}


def main():
    faulthandler.enable()
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=1000)
    ap.add_argument("--impl", default="fundem", choices=["fundem", "reference"])
    ap.add_argument("--n", type=int, default=262144)
    ap.add_argument("--footprint", type=int, nargs=2, default=[128, 128])
    ap.add_argument("--cpu-sample", type=int, default=2048)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--profile", action="store_true",
                    help="bracket the timed steps with cudaProfilerStart/Stop (for ncu --profile-from-start off)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision comparison")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint cost measurement")
    ap.add_argument("--adjoint-steps", type=int, default=20000)
    ap.add_argument("--no-autotune", action="store_true", help="keep the default narrow-phase launch shape")
    ap.add_argument("--no-graph", action="store_true", help="time plain launches instead of a K-step graph replay")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched calibration measurement")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip timing the reference's own CUDA build on the same state")
    ap.add_argument("--reference-gpu-steps", type=int, default=30)
    ap.add_argument("--reference-gpu-timeout", type=float, default=400.0)
    ap.add_argument("--settle-steps", type=int, default=24000, help="most settling steps of the workload")
    ap.add_argument("--pair-cache", type=int, default=-1, choices=[-1, 0, 1],
                    help="pair cache of the particle-particle list: -1 library default, 0 off, 1 on")
    ap.add_argument("--pair-skin", type=float, default=0.0, help="pair-cache skin in metres (0: default)")
    ap.add_argument("--batch-sims", type=int, default=256)
    ap.add_argument("--batch-steps", type=int, default=200)
    ap.add_argument("--batch-warmup", type=int, default=50)
    ap.add_argument("--batch-adjoint-sims", type=int, default=32)
    ap.add_argument("--batch-adjoint-steps", type=int, default=200)
    ap.add_argument("--error-steps", type=int, default=1000,
                    help="steps before the mixed-precision position error is measured")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if world > 1:
        import torch
        import torch.distributed as D
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        D.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
        dist = D
    try:
        if args.impl == "reference":
            run_reference(args, rank, world)
        else:
            run_fundem(args, rank, world, dist)
    finally:
        if dist:
            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
