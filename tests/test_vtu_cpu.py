"""The VTK XML writer of the drop-in headers (fundem_b200/kernel/VTUWriter.h):
a file written from known points, cells and arrays reads back unchanged
(inline base64 blocks with a 64-bit byte count).  No GPU."""
import os
import shutil
import subprocess

import numpy as np
import pytest

import vtu_read as V

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("g++") is None, reason="no host compiler")
def test_vtu_round_trip(tmp_path):
    src = tmp_path / "w.cpp"
    src.write_text(r'''
#include "kernel/VTUWriter.h"
#include <cstdio>
int main(int argc, char** argv) {
    // two triangles over four points, and one point cloud without cells
    std::vector<float> pts = {0.f, 0.f, 0.f, 1.f, 0.f, 0.f, 1.f, 1.f, 0.5f, -2.5f, 3.25f, 1e-7f};
    std::vector<int32_t> conn = {0, 1, 2, 0, 2, 3}, offs = {3, 6};
    std::vector<uint8_t> types = {5, 5};
    std::vector<int32_t> id = {7, 7, 8, -1};
    std::vector<float> vel = {1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12};
    std::vector<float> q = {1, 0, 0, 0, 0.5f, 0.5f, 0.5f, 0.5f, 0, 1, 0, 0, 0, 0, 1, 0};
    bool ok = fundem_vtu::write(argv[1], 0.125, 42, pts, conn, offs, types,
                                {fundem_vtu::array("particleID", 1, id), fundem_vtu::array("velocity", 3, vel),
                                 fundem_vtu::array("orientation", 4, q)});
    ok &= fundem_vtu::write(argv[2], 2.0, 7, std::vector<float>(pts.begin(), pts.begin() + 3), {}, {}, {}, {});
    // lengths 1, 2 and 3 bytes past the header exercise the base64 padding
    for (int n = 1; n <= 3; ++n) {
        std::vector<uint8_t> t(n, 0xAB);
        ok &= fundem_vtu::write(std::string(argv[3]) + std::to_string(n) + ".vtu", 0.0, 0, {0.f, 0.f, 0.f},
                                {0}, {1}, {1}, {fundem_vtu::array("bytes", 1, t)});
    }
    return ok ? 0 : 1;
}
''')
    exe = str(tmp_path / "w")
    subprocess.check_call(["g++", "-std=c++17", "-I", os.path.join(ROOT, "fundem_b200"), str(src), "-o", exe])
    a, b, c = tmp_path / "a.vtu", tmp_path / "b.vtu", tmp_path / "c"
    subprocess.check_call([exe, str(a), str(b), str(c)])
    m = V.read(a)
    assert m["n_points"] == 4 and m["n_cells"] == 2
    assert np.array_equal(m["points"].ravel(), np.array([0, 0, 0, 1, 0, 0, 1, 1, 0.5, -2.5, 3.25, 1e-7], np.float32))
    assert np.array_equal(m["connectivity"], [0, 1, 2, 0, 2, 3]) and np.array_equal(m["offsets"], [3, 6])
    assert np.array_equal(m["types"], [5, 5])
    assert np.array_equal(m["point_data"]["particleID"], [7, 7, 8, -1])
    assert m["point_data"]["velocity"].shape == (4, 3) and m["point_data"]["velocity"][3, 2] == 12
    assert m["point_data"]["orientation"].shape == (4, 4)
    assert m["field"]["TIME"] == np.float32(0.125) and m["field"]["STEP"] == 42
    p = V.read(b)
    assert p["n_points"] == 1 and p["n_cells"] == 0 and p["field"]["STEP"] == 7
    for n in (1, 2, 3):
        t = V.read(str(c) + f"{n}.vtu")
        assert np.array_equal(t["point_data"]["bytes"], np.full(n, 0xAB, np.uint8))
