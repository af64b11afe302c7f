"""Run an app written against the LSSolver call surface on the GPU: a sphere
dropped on a plane (tests/apps/sphere_drop.cpp), with and without an
addExternalForceTorque hook that launches its own CUDA kernel on the
solver's force array."""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
APPS = os.path.join(ROOT, "tests", "apps")


@pytest.fixture(scope="module")
def app(tmp_path_factory):
    from fundem_b200 import build
    d = tmp_path_factory.mktemp("app")
    return build.build_app([os.path.join(APPS, "sphere_drop.cpp"), os.path.join(APPS, "sphere_hover.cu")],
                           str(d / "sphere_drop")), d


def _run(app, *args):
    exe, d = app
    r = subprocess.run([exe, str(d / "out"), *args], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    vals = [float(v) for v in r.stdout.split()[-6:]]
    return np.array(vals[:3]), np.array(vals[3:]), d


def test_elastic_drop_conserves_energy(app):
    # r = 0.01, released at z = 0.05 with restitution 1 and no damping: after
    # the bounce g z + v^2 / 2 is back to g h0, within the integration error
    # of a contact resolved in about 14 steps (12 coincident pole nodes make
    # the contact stiffness 12 kn, dt = tc / 50)
    x, v, d = _run(app)
    g, h0 = 9.81, 0.05
    assert x[2] > 0.01  # above the plane, after the bounce
    assert v[2] > 0.0   # rising
    assert abs((g * x[2] + 0.5 * v @ v) - g * h0) < 1e-2 * g * h0
    frames = sorted(os.listdir(d / "out_phase1" / "LSParticle"))
    assert len(frames) >= 4 and frames[0].endswith(".vtu")


def test_hook_force_cancels_gravity(app):
    # The hook's force reaches the second half-kick of each step and, through
    # the force array, the first half-kick of the next.  The first half-kick
    # of the first step sees no force yet (LSSolver.h:1093-1107), so the
    # sphere keeps v = -g dt / 2 and sinks by that speed times the run time.
    x, v, _ = _run(app, "hover")
    g, h0, dt = 9.81, 0.05, 0.005 / 50.0
    steps = int(0.15 / dt) + 1 + 1
    assert abs(v[2] + 0.5 * g * dt) < 1e-12
    assert abs(v[0]) < 1e-15 and abs(v[1]) < 1e-15
    assert abs(x[2] - (h0 - steps * dt * 0.5 * g * dt)) < 1e-12


def test_device_getters_from_a_hook(tmp_path):
    """SolidInteraction's and VBondedInteraction's device getters
    (contactPoint(), masterID(), slaveID(), slidingSpring(),
    contactOverlap(), activated(), B1(), Un(), the bond frames, ...) read
    inside an addExternalForceTorque hook hold the same contacts and bonds as
    the host getters (tests/apps/view_check.cpp), at every step."""
    from fundem_b200 import build
    exe = build.build_app([os.path.join(APPS, "view_check.cpp")], str(tmp_path / "view_check"))
    r = subprocess.run([exe, str(tmp_path / "out")], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.split()[-3:-1] == ["views", "ok"]
    assert int(r.stdout.split()[-1]) > 100
