"""The LSSolver call surface (fundem_b200/kernel/): apps written against the
reference's kernel/LSSolver.h compile unchanged against it and link with
libfundem_b200.so.  No GPU needed."""
import os
import shutil
import subprocess

import pytest

from oracle.refpath import reference_path

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
APPS = os.path.join(ROOT, "tests", "apps")
CUDA_INC = "/usr/local/cuda/include"
REF_APP = reference_path("apps", "test", "LSSphereBouncing.cpp")


def _syntax(src, extra=()):
    cmd = ["g++", "-std=c++17", "-Wall", "-fsyntax-only", "-I", os.path.join(ROOT, "fundem_b200"), "-I", CUDA_INC,
           *extra, src]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


@pytest.mark.skipif(shutil.which("g++") is None, reason="no host compiler")
def test_own_app_compiles():
    _syntax(os.path.join(APPS, "sphere_drop.cpp"))


@pytest.mark.skipif(REF_APP is None or shutil.which("g++") is None,
                    reason="reference sources not present")
def test_reference_app_compiles_unchanged():
    """The reference's own sphere-bouncing app, as it lies in the reference
    tree, against these headers."""
    _syntax(REF_APP)


@pytest.mark.skipif(shutil.which("nvcc") is None, reason="no nvcc")
def test_app_links(tmp_path):
    from fundem_b200 import build
    exe = build.build_app([os.path.join(APPS, "sphere_drop.cpp"), os.path.join(APPS, "sphere_hover.cu")],
                          str(tmp_path / "sphere_drop"))
    assert os.path.exists(exe)
