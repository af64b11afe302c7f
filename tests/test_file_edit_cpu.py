"""The drop-in myFileEdit.h helpers (MKDIR, has*Ext, remove*Files), which
apps see through LSSolver.h, against the reference's header: the same
program built against each, run on the same directory tree (plain files with
each extension and with near misses, a directory and a link to a directory
named like frame files), prints the same results."""
import os
import shutil
import subprocess

import pytest

from oracle.refpath import reference_path

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_KERNEL = reference_path("kernel")
SRC = os.path.join(ROOT, "tests", "apps", "file_edit_check.cpp")

pytestmark = pytest.mark.skipif(shutil.which("g++") is None, reason="no host compiler")


def _tree(d):
    os.makedirs(d)
    for n in ["a.vtu", "b.vtu", "a.VTU", "a.vtu.bak", ".vtu", "x.vtm", "y.vti", "z.obj", "w.dat", "keep.txt"]:
        with open(os.path.join(d, n), "w") as f:
            f.write("x")
    os.makedirs(os.path.join(d, "frames.vtu"))          # a directory: kept
    with open(os.path.join(d, "frames.vtu", "in.vtu"), "w") as f:
        f.write("x")                                    # inside a subdirectory: kept
    os.makedirs(os.path.join(d, "real"))
    os.symlink(os.path.join(d, "real"), os.path.join(d, "link.vtu"))  # a link to a directory: removed


def _run(tmp_path, include_dir, tag):
    exe = str(tmp_path / f"check_{tag}")
    subprocess.check_call(["g++", "-O1", "-std=c++17", "-I", include_dir, SRC, "-o", exe])
    d = str(tmp_path / f"tree_{tag}")
    _tree(d)
    return subprocess.run([exe, d], capture_output=True, text=True, check=True).stdout


def test_file_helpers(tmp_path):
    ours = _run(tmp_path, os.path.join(ROOT, "fundem_b200", "kernel"), "ours")
    assert "vtu 4\n" in ours                # a.vtu, b.vtu, .vtu and the link
    assert "missing 0\n" in ours
    assert "  keep.txt\n" in ours and "  frames.vtu\n" in ours and "  a.VTU\n" in ours
    assert "mkdir 0 -1\n" in ours          # made, then already there
    if REF_KERNEL and os.path.isdir(REF_KERNEL):
        assert ours == _run(tmp_path, REF_KERNEL, "ref")
