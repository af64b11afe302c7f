"""Golden fixtures for the shape, packing and OBJ helpers.

The reference's helpers (kernel/helper/LevelSetObjectGenerator.h,
SpherePackingGenerator.h, OBJLoader.h) are header-only host code.
`make -C oracle helpers` compiles oracle/helpers_dump.cpp against them where
they lie; this script runs that program on the cases below and stores every
result in tests/golden/helpers.npz, together with the case list and the OBJ
text it read, so that a test can feed the same inputs to this library's
drop-in headers:

    python tests/golden/make_helper_fixtures.py

The OBJ input is synthetic: a torus written here with quads, a polygon face,
texture/normal index parts and negative indices.
"""
from __future__ import annotations

import math
import os
import struct
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
DUMP = os.path.join(ROOT, "oracle", "_ref", "helpers_dump")
OUT = os.path.join(HERE, "helpers.npz")

# {OBJ} is replaced by the path of the torus file
CASES = """\
SE ellipsoid 1.0 0.8 0.6 1.0 1.0 2 12 2
SE flatbox 0.4 1.0 0.8 0.4 1.6 3 12 2
SE sharp 0.42 1.0 0.83 0.1 1.0 1 12 1
SE pillow 1.0 1.0 1.0 1.0 0.5 2 10 3
SE blob 0.5 0.7 1.0 1.4 1.2 0 12 2
SP sphere 0.5 100 12 2
SP sphere12 0.25 12 8 1
BX box 1.0 0.7 2.0 12 2
CY drum -1.0 0.0 0.0 1.0 0.0 0.0 2.0 32 2 16 2
CY tilted 0.1 0.2 -0.5 0.3 -0.1 0.7 0.4 24 3 12 2
MS torus {OBJ} 0 12 2
MS torus_wall {OBJ} 1 8 1
PR regular 0.0 0.0 0.0 1.0 1.0 3.0 0.1
PH hex 0.0 0.0 0.0 1.0 1.0 1.0 0.07
PB box_random 0.0 0.0 0.0 1.0 1.0 2.0 300 0.03 0.08 12345 2000
PC drum_random -1.0 0.0 0.0 1.0 0.0 0.0 2.0 500 0.1 0.3 12345 2000
QR pack_regular 0.0 0.0 0.0 1.0 1.0 3.0 0.1
QH pack_hex -0.5 0.0 0.2 1.0 1.3 1.0 0.07
QB pack_random 1.0 2.0 3.0 0.0 0.0 0.0 400 0.02 0.09 777 500
QB pack_crowded 0.0 0.0 0.0 0.5 0.5 0.5 2000 0.03 0.05 12345 200
QB pack_thin 0.0 0.0 0.0 2.0 2.0 0.05 50 0.03 0.04 3 100
"""


def torus_obj(R=1.0, r=0.35, nu=16, nv=8):
    """A closed, non-convex mesh: quads around a torus; one row of quads is
    written as a single polygon strip fan, and some faces use negative indices
    and v/vt/vn tokens."""
    lines = ["# synthetic torus", "o torus"]
    for i in range(nu):
        a = 2 * math.pi * i / nu
        for j in range(nv):
            b = 2 * math.pi * j / nv
            x = (R + r * math.cos(b)) * math.cos(a)
            y = (R + r * math.cos(b)) * math.sin(a)
            z = r * math.sin(b)
            lines.append(f"v {x:.12e} {y:.12e} {z:.12e}")
    lines.append("vt 0 0")
    lines.append("vn 0 0 1")
    nverts = nu * nv

    def vid(i, j):
        return (i % nu) * nv + (j % nv) + 1

    for i in range(nu):
        for j in range(nv):
            q = [vid(i, j), vid(i + 1, j), vid(i + 1, j + 1), vid(i, j + 1)]
            k = (i * nv + j) % 4
            if k == 0:
                lines.append("f " + " ".join(str(t) for t in q))
            elif k == 1:
                lines.append("f " + " ".join(f"{t}/1/1" for t in q))
            elif k == 2:
                lines.append("f " + " ".join(f"{t - nverts - 1}//1" for t in q))
            else:
                lines.append(f"f {q[0]} {q[1]} {q[2]}")
                lines.append(f"f {q[0]}/1 {q[2]}/1 {q[3]}/1")
    return "\n".join(lines) + "\n"


def read_records(path):
    out = {}
    with open(path, "rb") as f:
        data = f.read()
    p = 0
    while p < len(data):
        (n,) = struct.unpack_from("<i", data, p)
        p += 4
        name = data[p:p + n].decode()
        p += n
        typ, count = struct.unpack_from("<iq", data, p)
        p += 12
        dt = np.float64 if typ == 0 else np.int32
        size = count * (8 if typ == 0 else 4)
        out[name] = np.frombuffer(data[p:p + size], dtype=dt).copy()
        p += size
    return out


def run_dump(exe, cases, obj_text, nogrid=False, env=None):
    """Write the torus, run `exe` on the cases and return its records."""
    with tempfile.TemporaryDirectory() as d:
        obj = os.path.join(d, "torus.obj")
        with open(obj, "w") as f:
            f.write(obj_text)
        out = os.path.join(d, "out.bin")
        args = [exe, out] + (["nogrid"] if nogrid else [])
        subprocess.run(args, input=cases.replace("{OBJ}", obj), text=True, check=True, env=env,
                       stdout=subprocess.DEVNULL)
        return read_records(out)


def main():
    if not os.path.exists(DUMP):
        subprocess.check_call(["make", "-C", os.path.join(ROOT, "oracle"), "helpers"])
    obj_text = torus_obj()
    rec = run_dump(DUMP, CASES, obj_text)
    np.savez_compressed(OUT, __cases__=np.array(CASES), __obj__=np.array(obj_text), **rec)
    print(f"{OUT}: {len(rec)} arrays, {os.path.getsize(OUT)} bytes")


if __name__ == "__main__":
    sys.exit(main())
