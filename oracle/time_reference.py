"""Time the reference's own CUDA build against this library on one workload.

    python oracle/time_reference.py N FX FY [STEPS]
    python oracle/time_reference.py pour [STEPS]

Builds the bonded periodic column with N particles on an FX x FY footprint
(fundem_b200.workloads.bonded_column, on the GPU), or the 1,000-particle
pour in a box of six walls (fundem_b200.scenario.pour, the small pour's
shape), times 100 steps of this library (1,000 for the pour) from that state, then writes the same scenario for the reference
(oracle.scenario_io.write_reference_scenario) and runs oracle/_ref/ref_driver
in timing mode over STEPS steps.  The driver reports the wall time between
the hooks of steps 20 and STEPS - 10, after a device synchronisation at each
end; no output frame falls in that window (the reference writes VTU frames
at the start and end of solve).  The scenario and the reference's VTU output
go to a scratch directory under /tmp, removed afterwards; a JSON summary goes
to the directory named by the environment variable FUNDEM_TIMING_OUT, else to
the current directory.

Measurement infrastructure: needs a GPU and oracle/_ref/ref_driver built by
oracle/Makefile from the reference sources.
"""
import json
import os
import shutil
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def main():
    import torch
    from fundem_b200 import workloads
    from oracle import scenario_io

    if sys.argv[1] == "pour":
        import fundem_b200 as F
        from fundem_b200 import scenario as S
        sc = S.pour(n=1000, n_templates=4, seed=0)
        n, fx, fy, info = 1000, 0, 0, {"workload": "pour"}
        steps_ref = int(sys.argv[2]) if len(sys.argv) > 2 else 2000
        sim = F.Simulation.from_scenario(sc)
        sim.detect()
        ours_steps = 1000
    else:
        n, fx, fy = int(sys.argv[1]), int(sys.argv[2]), int(sys.argv[3])
        steps_ref = int(sys.argv[4]) if len(sys.argv) > 4 else 50
        sim, sc, info = workloads.bonded_column(n=n, footprint=(fx, fy), seed=1)
        ours_steps = 100
    sim.set_records(False)
    sim.step(20)
    sim.sync()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    sim.step(ours_steps)
    e1.record()
    torch.cuda.synchronize()
    sim.sync()
    ours = e0.elapsed_time(e1) / ours_steps
    print(f"fundem_b200: {ours:.4f} ms/step at n={n} (steps 20..{20 + ours_steps})", flush=True)
    sim.close()
    torch.cuda.empty_cache()

    out = tempfile.mkdtemp(prefix=f"fundem_ref_{n}_")
    try:
        path = os.path.join(out, "scenario.bin")
        scenario_io.write_reference_scenario(sc, path, steps_ref)
        t0 = time.time()
        r = subprocess.run([os.path.join(ROOT, "oracle", "_ref", "ref_driver"), path, out, "timing", "20",
                            str(steps_ref - 10)], capture_output=True, text=True)
        print("reference rc", r.returncode, "wall", round(time.time() - t0, 1), "s", flush=True)
        print(r.stdout[-600:])
        meta = {}
        with open(os.path.join(out, "meta.txt")) as f:
            for line in f:
                k, v = line.split(None, 1)
                meta[k] = v.strip()
    finally:
        shutil.rmtree(out, ignore_errors=True)
    ref = 1e3 * float(meta["window_seconds"]) / float(meta["window_steps"])
    res = dict(particles=n, footprint=[fx, fy], info=info, fundem_ms_per_step=ours, reference_ms_per_step=ref,
               reference_window=[20, steps_ref - 10], ratio=ref / ours)
    print(json.dumps(res), flush=True)
    dst = os.environ.get("FUNDEM_TIMING_OUT", ".")
    with open(os.path.join(dst, f"reference_timing_{n}.json"), "w") as f:
        json.dump(res, f, default=str)
    return r.returncode


if __name__ == "__main__":
    sys.exit(main())
