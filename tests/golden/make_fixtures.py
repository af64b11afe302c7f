"""Generate the golden fixtures that pin parity to the reference.

Two steps, because the reference is CUDA-only:

1. On a GPU machine (the reference driver must already be built by
   `make -C oracle ref`, which needs the reference sources):

       python tests/golden/make_fixtures.py run --out <dir>

   writes each parity scenario (tests/parity_cases.py) for the driver, runs
   the reference's own build on it and leaves the dumps in <dir>/<case>/.

2. Anywhere:

       python tests/golden/make_fixtures.py collect --src <dir>

   reduces the dumps to tests/golden/<case>.npz: the per-step particle
   state, every contact list (all five kinds), the bond state, and the
   SHA-256 of the scenario file so a test can check it rebuilt the same
   inputs.
"""
from __future__ import annotations

import argparse
import glob
import hashlib
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import parity_cases as PC  # noqa: E402
from oracle import scenario_io as SIO  # noqa: E402

DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_driver")


def scenario_bytes(name):
    import tempfile
    sc = PC.CASES[name]()
    n, dumps = PC.REF_STEPS[name]
    with tempfile.NamedTemporaryFile(suffix=".bin", delete=False) as f:
        path = f.name
    SIO.write_reference_scenario(sc, path, n, dumps)
    with open(path, "rb") as f:
        data = f.read()
    os.unlink(path)
    return data


def run(out, cases):
    # the reference resolves relative output directories against the
    # executable's location (LSSolver.h:638-644): pass absolute paths
    out = os.path.abspath(out)
    os.makedirs(out, exist_ok=True)
    for name in cases:
        d = os.path.join(out, name)
        os.makedirs(d, exist_ok=True)
        path = os.path.join(d, "scenario.bin")
        with open(path, "wb") as f:
            f.write(scenario_bytes(name))
        print("reference:", name, flush=True)
        subprocess.check_call([DRIVER, path, d])


def collect(src, cases):
    for name in cases:
        d = os.path.join(src, name)
        with open(os.path.join(d, "scenario.bin"), "rb") as f:
            sha = hashlib.sha256(f.read()).hexdigest()
        out = {"scenario_sha256": np.array(sha)}
        steps = []
        for p in sorted(glob.glob(os.path.join(d, "dump_*.bin"))):
            dump = SIO.read_dump(p)
            s = dump["step"]
            steps.append(s)
            for k in ("pos", "vel", "angvel", "quat", "force", "torque", "wall_pos", "wall_quat"):
                out[f"s{s}_{k}"] = dump[k]
            for kind in SIO.KINDS + SIO.SECTOR_KINDS:
                if kind not in dump:
                    continue
                for k, v in dump[kind].items():
                    out[f"s{s}_{kind}_{k}"] = v
            for k, v in dump["bonds"].items():
                out[f"s{s}_bond_{k}"] = v
        out["steps"] = np.array(steps, dtype=np.int64)
        g = SIO.read_geometry(os.path.join(d, "geometry.bin"))
        for k, v in g.items():
            out[f"geo_{k}"] = v
        with open(os.path.join(d, "meta.txt")) as f:
            out["meta"] = np.array(f.read())
        dst = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(dst, **out)
        print("wrote", dst, os.path.getsize(dst), "bytes")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("mode", choices=["run", "collect", "sha"])
    ap.add_argument("--out", default="ref_dumps")
    ap.add_argument("--src", default="ref_dumps")
    ap.add_argument("--cases", nargs="*", default=list(PC.CASES))
    a = ap.parse_args()
    if a.mode == "run":
        run(a.out, a.cases)
    elif a.mode == "collect":
        collect(a.src, a.cases)
    else:
        for name in a.cases:
            print(name, hashlib.sha256(scenario_bytes(name)).hexdigest())


if __name__ == "__main__":
    main()
