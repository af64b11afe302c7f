"""Build libfundem_b200.so in-tree (nvcc, sm_100a).

    python -m fundem_b200.build

The library lands in fundem_b200/_lib/ next to this file; the Python
bindings load it from there and nowhere else.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libfundem_b200.so")
SOURCES = ["fd_kernels.cu", "fd_adjoint.cu", "fd_api.cu", "fd_levelset.cu"]
# per-source flags: the grid generator rounds every add and multiply on its own
SOURCE_FLAGS = {"fd_levelset.cu": ["-fmad=false"]}
HEADERS = ["fd_internal.cuh", "fd_kernels.cuh", "fd_adjoint.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC = os.environ.get("NVCC", "nvcc")
# extra compiler definitions, e.g. FUNDEM_NVCC_DEFS="-DFD_NARROW_MIN_BLOCKS=1"
EXTRA = os.environ.get("FUNDEM_NVCC_DEFS", "").split()


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(ROOT, "include", "fundem_b200.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    objs = []
    for src in SOURCES:
        obj = os.path.join(LIBDIR, src.replace(".cu", ".o"))
        cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
               "-I", os.path.join(ROOT, "include"), *EXTRA, *SOURCE_FLAGS.get(src, []), "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd))
        subprocess.check_call(cmd)
        objs.append(obj)
    tmp = LIB + ".tmp"
    subprocess.check_call([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs])
    os.replace(tmp, LIB)
    for o in objs:
        os.remove(o)
    return LIB


KERNEL_HEADERS = HERE  # the directory holding kernel/LSSolver.h and the value types


def build_app(sources, output, include_dirs=(), verbose=False) -> str:
    """Build an app written against the LSSolver call surface (kernel/LSSolver.h)
    into an executable linked with libfundem_b200.so: .cpp sources go through
    the host compiler, .cu sources through nvcc for sm_100a."""
    build()
    cmd = [NVCC, *ARCH, "-O2", "-std=c++17", "-I", KERNEL_HEADERS, "-I", os.path.join(ROOT, "include")]
    for d in include_dirs:
        cmd += ["-I", d]
    cmd += list(sources) + ["-L", LIBDIR, "-lfundem_b200", "-Xlinker", "-rpath," + LIBDIR, "-o", output]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    return output


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
