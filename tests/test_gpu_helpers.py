"""Level-set grids evaluated on the GPU (fundem_levelset_grid, behind
LevelSetObject::Base::buildGrid) against the reference helpers' own grids
(tests/golden/helpers.npz), and two apps that use the helper namespaces end
to end: superellipsoids in a turning CylinderWall drum, and OBJ-mesh
particles falling into a BoxWall."""
import os
import time

import numpy as np
import pytest

from golden import make_helper_fixtures as MF

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
APPS = os.path.join(ROOT, "tests", "apps")
# FP64 grid values may differ from the host build where CUDA's pow (the
# superellipsoid) rounds differently from the host library; everything else
# is the same sequence of IEEE operations
GRID_ATOL = 1e-12


@pytest.fixture(scope="module")
def golden():
    z = np.load(os.path.join(ROOT, "tests", "golden", "helpers.npz"))
    return {k: z[k] for k in z.files}


@pytest.fixture(scope="module")
def dump_exe(tmp_path_factory, fundem):
    from fundem_b200 import build
    exe = str(tmp_path_factory.mktemp("helpers_gpu") / "helpers_dump")
    return build.build_app([os.path.join(ROOT, "oracle", "helpers_dump.cpp")], exe)


def _kind(golden, name):
    for line in str(golden["__cases__"]).splitlines():
        parts = line.split()
        if parts and parts[1] == name:
            return parts[0], parts[2:]
    raise KeyError(name)


def test_gpu_grids_match_reference(dump_exe, golden):
    rec = MF.run_dump(dump_exe, str(golden["__cases__"]), str(golden["__obj__"]))
    assert sorted(rec) == sorted(k for k in golden if not k.startswith("__"))
    report = []
    for k, v in rec.items():
        ref = golden[k]
        assert v.shape == ref.shape, k
        if not k.endswith("/sdf"):
            assert np.array_equal(v, ref), k
            continue
        diff = np.abs(v - ref)
        exact = np.count_nonzero(diff == 0) / diff.size
        report.append((k, float(diff.max()), exact))
        kind, _ = _kind(golden, k.split("/")[0])
        assert diff.max() <= GRID_ATOL * max(1.0, float(np.abs(ref).max())), (k, diff.max())
        if kind in ("SP", "BX", "CY"):
            # no transcendental function on these paths: bit for bit
            assert exact == 1.0, (k, exact)
        if kind == "MS":
            # the winding-number sign must agree everywhere
            assert np.array_equal(np.sign(v), np.sign(ref)), k
    print("\n".join(f"{k}: max |diff| {d:.3e}, bit-exact {e:.4f}" for k, d, e in report))


def test_python_binding_matches(golden, fundem):
    """fundem_b200.levelset_grid with the layout of fundem_b200.grid_layout."""
    for line in str(golden["__cases__"]).splitlines():
        c = line.split()
        kind, name = c[0], c[1]
        if kind == "SE":
            rx, ry, rz, ee, en = map(float, c[2:7])
            args = ("superellipsoid", [rx, ry, rz, ee, en])
            lo, hi = [-rx, -ry, -rz], [rx, ry, rz]
        elif kind == "BX":
            lx, ly, lz = map(float, c[2:5])
            args = ("box", [lx, ly, lz])
            lo, hi = [-lx / 2, -ly / 2, -lz / 2], [lx / 2, ly / 2, lz / 2]
        elif kind == "SP":
            r = float(c[2])
            args = ("sphere", [r])
            lo, hi = [-r] * 3, [r] * 3
        else:
            continue
        res, pad = int(c[-2]), int(c[-1])
        h = max(b - a for a, b in zip(lo, hi)) / res
        origin, size = fundem.grid_layout(lo, hi, h, pad)
        sdf = fundem.levelset_grid(*args, origin, h, size, positive_inside=(kind == "BX"))
        ref = golden[name + "/sdf"]
        assert np.abs(sdf - ref).max() <= GRID_ATOL, name


def test_mesh_grid_throughput(golden, fundem):
    """A 65 x 65 x 20 grid of the torus mesh and a 129^3 superellipsoid grid:
    a sanity check on speed, printed for the record."""
    v = golden["torus/vertices"].reshape(-1, 3)
    t = golden["torus/triangles"].reshape(-1, 3)
    h = 2.8 / 60
    origin, size = fundem.grid_layout(v.min(0), v.max(0), h, 2)
    fundem.levelset_grid("mesh", None, origin, h, size, vertices=v, triangles=t)
    t0 = time.perf_counter()
    sdf = fundem.levelset_grid("mesh", None, origin, h, size, vertices=v, triangles=t)
    t_mesh = time.perf_counter() - t0
    n_mesh = int(np.prod(size))
    assert np.isfinite(sdf).all() and (sdf < 0).any() and (sdf > 0).any()
    origin, size = fundem.grid_layout([-1, -1, -1], [1, 1, 1], 2.0 / 124, 2)
    t0 = time.perf_counter()
    sdf = fundem.levelset_grid("superellipsoid", [1, 1, 1, 0.5, 0.5], origin, 2.0 / 124, size)
    t_se = time.perf_counter() - t0
    print(f"\nmesh {len(t)} triangles x {n_mesh} nodes: {t_mesh * 1e3:.1f} ms; "
          f"superellipsoid {int(np.prod(size))} nodes: {t_se * 1e3:.1f} ms")


def _state(path):
    return np.loadtxt(path, ndmin=2)


def test_drum_app(tmp_path, fundem):
    """Settle superellipsoids in a closed drum, then turn the drum at pi rad/s
    about its axis: everything stays inside, and the contents pick up angular
    momentum about the axis in the drum's sense."""
    from fundem_b200 import build
    import subprocess
    exe = build.build_app([os.path.join(APPS, "drum_rolling.cpp")], str(tmp_path / "drum_rolling"))
    out = tmp_path / "drum"
    r = subprocess.run([exe, str(out), "40"], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "LSSolver" not in r.stderr, r.stderr
    for phase in (0, 1):
        s = _state(out / f"state_{phase}.txt")
        assert np.isfinite(s).all()
        x, v, m = s[:, 0:3], s[:, 3:6], s[:, 6]
        assert len(s) >= 10
        assert np.all(np.abs(x[:, 0]) < 0.5 + 1e-6)
        assert np.all(np.hypot(x[:, 1], x[:, 2]) < 1.0)
        Lx = np.sum(m * (x[:, 1] * v[:, 2] - x[:, 2] * v[:, 1]))
        # angular momentum of the same bodies turning rigidly with the drum
        rigid = np.sum(m * (x[:, 1] ** 2 + x[:, 2] ** 2)) * np.pi
        if phase == 1:
            assert Lx > 0.2 * rigid, (Lx, rigid)
        print(f"phase {phase}: L_x {Lx:.3f}, rigid co-rotation {rigid:.3f}")
    _check_drum_frames(tmp_path / "drum_phase2", _state(out / "state_1.txt"))


def _check_drum_frames(d, state):
    """The last frame of the turning phase, as LSSolver::solve writes it: the
    particles' surface meshes and centres, the drum's mesh, and the particle
    and wall contacts."""
    import vtu_read as V
    last = sorted(os.listdir(d / "LSParticle"))[-1][-8:]  # NNNN.vtu
    centres = V.read(d / "LSParticle" / ("Particle_" + last))
    assert centres["n_points"] == len(state)
    assert np.allclose(centres["points"], state[:, :3], rtol=0, atol=1e-6)
    assert np.allclose(centres["point_data"]["velocity"], state[:, 3:6], rtol=1e-6, atol=1e-6)
    assert centres["point_data"]["orientation"].shape == (len(state), 4)
    mesh = V.read(d / "LSParticle" / ("LSObjectMesh_" + last))
    # subdivision level 3: 642 nodes and 1280 triangles per particle
    assert mesh["n_points"] == 642 * len(state) and mesh["n_cells"] == 1280 * len(state)
    assert np.all(mesh["types"] == 5) and mesh["offsets"][-1] == 3 * mesh["n_cells"]
    pid = mesh["point_data"]["particleID"]
    assert np.array_equal(pid, np.repeat(np.arange(len(state)), 642))
    # every node lies within its body's reach of the body's centre
    reach = np.linalg.norm(mesh["points"] - centres["points"][pid], axis=1)
    assert reach.max() < 0.3 and reach.min() > 0.0
    wall = V.read(d / "Wall" / ("LSObjectMesh_" + last))
    # 96 segments, 2 axial segments: 3 rings and 2 cap centres; 2 x 96 x 2 side and 2 x 96 cap triangles
    assert wall["n_points"] == 3 * 96 + 2 and wall["n_cells"] == 4 * 96 + 2 * 96
    for sub in ("LSParticleInteraction", "LSParticle-WallInteraction"):
        c = V.read(d / sub / ("LSInteraction_" + last))
        assert c["n_points"] > 0, sub
        n = c["point_data"]["contactNormal"]
        assert np.allclose(np.linalg.norm(n, axis=1), 1.0, atol=1e-5), sub
        assert np.all(np.hypot(c["points"][:, 1], c["points"][:, 2]) < 1.0 + 1e-3), sub
        assert np.all(c["point_data"]["normalElasticEnergy"] >= 0), sub


def test_mesh_falling_app(tmp_path, fundem):
    """Copies of an OBJ torus dropped into a box fall and stay inside it."""
    from fundem_b200 import build
    import subprocess
    exe = build.build_app([os.path.join(APPS, "mesh_falling.cpp")], str(tmp_path / "mesh_falling"))
    obj = tmp_path / "torus.obj"
    obj.write_text(MF.torus_obj(R=0.1, r=0.035))
    out = tmp_path / "box"
    r = subprocess.run([exe, str(out), str(obj)], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "LSSolver" not in r.stderr, r.stderr
    s = _state(out / "state.txt")
    assert len(s) >= 8 and np.isfinite(s).all()
    x = s[:, 0:3]
    assert np.all((x > -1e-6) & (x < np.array([1.0, 1.0, 2.0]) + 1e-6))
    # the lattice started at mean height 1.0; after 0.5 s the copies have fallen
    assert x[:, 2].mean() < 0.8
