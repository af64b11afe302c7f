"""The drop-in HostDeviceArray1D (myHostDeviceArray.h), which apps see
through LSSolver.h, against the reference's header: a program exercising the
host side (pushes, inserts, erases, resizes, moves) built against each
prints the same.  The device side (stream-ordered allocation and copies) has
no GPU here; it makes the reference's calls in the same order."""
import os
import shutil
import subprocess

import pytest

from oracle.refpath import reference_path

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_KERNEL = reference_path("kernel")
SRC = os.path.join(ROOT, "tests", "apps", "host_array_check.cpp")
CUDA = "/usr/local/cuda"

pytestmark = pytest.mark.skipif(shutil.which("g++") is None or not os.path.isdir(CUDA),
                                reason="no host compiler or CUDA headers")


def _run(tmp_path, include_dir, tag):
    exe = str(tmp_path / f"check_{tag}")
    subprocess.check_call(["g++", "-O1", "-std=c++17", "-I", include_dir, "-I", os.path.join(CUDA, "include"), SRC,
                           "-L", os.path.join(CUDA, "lib64"), "-lcudart", "-Wl,-rpath," + os.path.join(CUDA, "lib64"),
                           "-o", exe])
    return subprocess.run([exe], capture_output=True, text=True, check=True).stdout


def test_host_side(tmp_path):
    ours = _run(tmp_path, os.path.join(ROOT, "fundem_b200", "kernel"), "ours")
    assert "insert host 7 device 0 gb 0.000: 0 1.5 -1 3 4.5 6 9 ptr 0\n" in ours
    assert "moved-from host 0 " in ours and "moved-to host 3 " in ours
    if REF_KERNEL and os.path.isdir(REF_KERNEL):
        assert ours == _run(tmp_path, REF_KERNEL, "ref")
