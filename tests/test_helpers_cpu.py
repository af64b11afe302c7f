"""The helper namespaces of the drop-in headers (LevelSetObject::,
SpherePacking::, OBJLoader:: in fundem_b200/kernel/helper/) against golden
fixtures made by the reference's own helpers (tests/golden/helpers.npz,
tests/golden/make_helper_fixtures.py).  No GPU: the surface meshes, packings
and OBJ parsing are host code, and the grids are evaluated here through the
host path the headers take for user-derived shape classes.  The GPU grids are
covered by test_gpu_helpers.py."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from oracle.refpath import reference_path, reference_root

from golden import make_helper_fixtures as MF

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
APPS = os.path.join(ROOT, "tests", "apps")
CUDA_INC = "/usr/local/cuda/include"
REF_ROOT = reference_root()
REF_TUTORIAL = reference_path("apps", "tutorial")

needs_gxx = pytest.mark.skipif(shutil.which("g++") is None, reason="no host compiler")


@pytest.fixture(scope="module")
def golden():
    z = np.load(os.path.join(ROOT, "tests", "golden", "helpers.npz"))
    return {k: z[k] for k in z.files}


@pytest.fixture(scope="module")
def dump_exe(tmp_path_factory, fundem):
    """oracle/helpers_dump.cpp built against this library's headers (host
    compiler; linked with libfundem_b200.so, whose GPU entry is not called)."""
    from fundem_b200 import build
    exe = str(tmp_path_factory.mktemp("helpers") / "helpers_dump")
    cmd = ["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "fundem_b200"), "-I", os.path.join(ROOT, "include"),
           "-I", CUDA_INC, os.path.join(ROOT, "oracle", "helpers_dump.cpp"), "-L", build.LIBDIR, "-lfundem_b200",
           "-Wl,-rpath," + build.LIBDIR, "-o", exe]
    subprocess.check_call(cmd)
    return exe


def _records(exe, golden, mode):
    cases = str(golden["__cases__"])
    obj = str(golden["__obj__"])
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "torus.obj")
        with open(path, "w") as f:
            f.write(obj)
        out = os.path.join(d, "out.bin")
        subprocess.run([exe, out, mode], input=cases.replace("{OBJ}", path), text=True, check=True,
                       stdout=subprocess.DEVNULL)
        return MF.read_records(out)


@needs_gxx
def test_meshes_and_packings_bit_exact(dump_exe, golden):
    """Surface meshes of every shape (vertex order included), the OBJ mesh,
    the four SpherePacking:: packings and the five SpherePack (kernel/Packing.h)
    packings equal the reference's, bit for bit."""
    rec = _records(dump_exe, golden, "nogrid")
    assert len(rec) == 42
    for k, v in rec.items():
        assert v.dtype == golden[k].dtype and v.shape == golden[k].shape, k
        assert np.array_equal(v, golden[k]), k


@needs_gxx
def test_host_grids_bit_exact(dump_exe, golden):
    """Grid layout and values through the host evaluation path, every shape
    (including the mesh's closest-triangle distance and winding-number sign)."""
    rec = _records(dump_exe, golden, "host")
    grids = [k for k in rec if k.endswith("/sdf")]
    assert len(grids) == 12
    for k, v in rec.items():
        assert np.array_equal(v, golden[k]), k


def test_grid_layout_matches(golden, fundem):
    """fundem_b200.grid_layout lays the grid out as Base::buildGrid does."""
    cases = [ln.split() for ln in str(golden["__cases__"]).splitlines()]
    for c in cases:
        kind, name = c[0], c[1]
        if kind == "SE":
            rx, ry, rz = map(float, c[2:5])
            lo, hi = [-rx, -ry, -rz], [rx, ry, rz]
        elif kind == "BX":
            lx, ly, lz = map(float, c[2:5])
            lo, hi = [-lx / 2, -ly / 2, -lz / 2], [lx / 2, ly / 2, lz / 2]
        elif kind == "SP":
            r = float(c[2])
            lo, hi = [-r] * 3, [r] * 3
        else:
            continue
        res, pad = int(c[-2]), int(c[-1])
        h = max(b - a for a, b in zip(lo, hi)) / res
        origin, size = fundem.grid_layout(lo, hi, h, pad)
        assert np.array_equal(origin, golden[name + "/origin"]), name
        assert np.array_equal(size, golden[name + "/size"]), name
        assert golden[name + "/spacing"][0] == h


@pytest.mark.skipif(REF_ROOT is None, reason="reference sources absent")
@needs_gxx
def test_fixtures_reproduce_from_reference(tmp_path, golden):
    """The committed fixtures are what the reference's helpers produce now."""
    exe = str(tmp_path / "ref_helpers_dump")
    subprocess.check_call(["g++", "-O3", "-DNDEBUG", "-std=c++17", "-I", REF_ROOT, "-I", os.path.join(REF_ROOT, "kernel"),
                           "-I", CUDA_INC, os.path.join(ROOT, "oracle", "helpers_dump.cpp"), "-o", exe])
    rec = MF.run_dump(exe, str(golden["__cases__"]), str(golden["__obj__"]))
    assert sorted(rec) == sorted(k for k in golden if not k.startswith("__"))
    for k, v in rec.items():
        assert np.array_equal(v, golden[k]), k


@needs_gxx
def test_obj_loader_errors(tmp_path, fundem):
    """Malformed OBJ files give false and empty arrays; polygons are fanned and
    negative indices count back from the last vertex."""
    src = tmp_path / "obj_errors.cpp"
    src.write_text(r'''
#include "kernel/helper/OBJLoader.h"
#include <cstdio>
int main(int argc, char** argv) {
    const char* files[] = {"ok.obj", "zero.obj", "range.obj", "short.obj", "missing.obj", "badv.obj"};
    for (const char* f : files) {
        std::vector<double3> v; std::vector<int3> t;
        const bool ok = OBJLoader::loadOBJMesh(f, v, t, argc, argv, false);
        std::printf("%s %d %zu %zu", f, ok ? 1 : 0, v.size(), t.size());
        for (const int3& x : t) std::printf(" %d,%d,%d", x.x, x.y, x.z);
        std::printf("\n");
    }
    return 0;
}
''')
    verts = "v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nv 0 0 1\n"
    (tmp_path / "ok.obj").write_text("# c\n\n" + verts + "f 1 2 3 4 5\nf -1/2/3 -2//1 -3\n")
    (tmp_path / "zero.obj").write_text(verts + "f 0 1 2\n")
    (tmp_path / "range.obj").write_text(verts + "f 1 2 9\n")
    (tmp_path / "short.obj").write_text(verts + "f 1 2\n")
    (tmp_path / "badv.obj").write_text("v 0 0\n")
    exe = str(tmp_path / "obj_errors")
    subprocess.check_call(["g++", "-std=c++17", "-I", os.path.join(ROOT, "fundem_b200"), "-I", CUDA_INC, str(src),
                           "-o", exe])
    out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.splitlines()
    assert out[0] == "ok.obj 1 5 4 0,1,2 0,2,3 0,3,4 4,3,2"
    for line in out[1:]:
        assert line.split()[1:] == ["0", "0", "0"], line


@pytest.mark.skipif(REF_TUTORIAL is None or shutil.which("g++") is None,
                    reason="reference sources not present")
@pytest.mark.parametrize("app", ["LSParticleFalling.cpp", "LSParticleRolling.cpp"])
def test_reference_tutorials_compile_unchanged(app):
    """The reference's tutorial apps, as they lie in the reference tree, compile
    against these headers (solver, helper namespaces, value types)."""
    cmd = ["g++", "-std=c++17", "-fsyntax-only", "-I", os.path.join(ROOT, "fundem_b200"),
           "-I", os.path.join(ROOT, "include"), "-I", CUDA_INC, os.path.join(REF_TUTORIAL, app)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
