"""The reference's own sphere-bouncing app (apps/test/LSSphereBouncing.cpp),
unchanged, run twice on the GPU: built against the reference's headers and
CUDA kernels, and built against the drop-in headers (fundem_b200/kernel) and
linked with libfundem_b200.so.  Both executables come from the oracle recipe
(`make -C oracle apps REF_ROOT=...`), which compiles the app where it lies in
the reference tree; nothing here reads the reference sources.

The app drops a 1 cm sphere from 1 m onto a plane wall (no damping, no
friction, dt = 1e-4 s, 2 s, 200 frames) and writes its frames under
LSSphereBouncing_phase1/ beside the executable.  Each binary runs from its
own copy in a temporary directory, and the particle-centre frames
(LSParticle/Particle_NNNN.vtu) are compared: the same frames, TIME and STEP,
positions to 1e-6 m and velocities to 1e-5 m/s (the frames store float32)."""
import glob
import os
import shutil
import subprocess

import numpy as np
import pytest

import vtu_read

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
APPDIR = os.path.join(ROOT, "oracle", "_ref", "apps")
LIBDIR = os.path.join(ROOT, "fundem_b200", "_lib")
APP = "LSSphereBouncing"


def _run(variant, tmp):
    exe = os.path.join(APPDIR, f"{APP}_{variant}")
    if not os.path.exists(exe):
        pytest.skip(f"{exe} not built (make -C oracle apps needs the reference sources)")
    d = tmp / variant
    d.mkdir()
    local = str(d / APP)
    shutil.copy2(exe, local)
    env = dict(os.environ)
    env["LD_LIBRARY_PATH"] = LIBDIR + os.pathsep + env.get("LD_LIBRARY_PATH", "")
    r = subprocess.run([local], cwd=str(d), env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, (variant, r.stdout[-2000:], r.stderr[-2000:])
    files = sorted(glob.glob(str(d / f"{APP}_phase1" / "LSParticle" / "Particle_*.vtu")))
    assert files, (variant, "no frames written", r.stdout[-1000:])
    return files


def test_sphere_bouncing_app_matches_reference_build(tmp_path):
    import fundem_b200
    fundem_b200.lib()   # the in-tree library the drop-in binary links
    ref = _run("ref", tmp_path)
    ours = _run("fundem", tmp_path)
    assert [os.path.basename(f) for f in ours] == [os.path.basename(f) for f in ref]
    dx = dv = 0.0
    zmin = np.inf
    for a, b in zip(ours, ref):
        fa, fb = vtu_read.read(a), vtu_read.read(b)
        assert fa["n_points"] == fb["n_points"] == 1
        assert fa["field"]["STEP"] == fb["field"]["STEP"], a
        assert fa["field"]["TIME"] == pytest.approx(fb["field"]["TIME"], rel=1e-6, abs=1e-9), a
        dx = max(dx, float(np.abs(fa["points"].astype(np.float64) - fb["points"]).max()))
        dv = max(dv, float(np.abs(fa["point_data"]["velocity"].astype(np.float64)
                                  - fb["point_data"]["velocity"]).max()))
        zmin = min(zmin, float(fb["points"][0, 2]))
    # the sphere reached the wall (centre within one radius of the plane)
    assert zmin < 0.0101, zmin
    assert dx <= 1e-6, dx
    assert dv <= 1e-5, dv
    print(f"{len(ref)} frames, max |dx| {dx:.3e} m, max |dv| {dv:.3e} m/s, lowest centre {zmin:.5f} m")
