"""CPU checks of the drop-in boundary: the library builds for sm_100a, loads
without a GPU, and exports every entry point include/fundem_b200.h declares."""
import os
import re

import pytest

from conftest import ROOT


def declared_functions():
    with open(os.path.join(ROOT, "include", "fundem_b200.h")) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fundem_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_bound_symbols(fundem):
    assert declared_functions() == sorted(fundem.EXPORTS)


def test_library_exports_every_declared_symbol(fundem):
    L = fundem.lib()
    for name in declared_functions():
        assert hasattr(L, name), name
    assert L.fundem_version().decode().startswith("fundem_b200")


def test_status_strings(fundem):
    L = fundem.lib()
    for code in range(6):
        assert L.fundem_status_string(code)


def test_library_is_built_for_sm100a(fundem):
    # cuobjdump-free check: nvcc was asked for sm_100a only
    from fundem_b200 import build
    assert "arch=compute_100a,code=sm_100a" in " ".join(build.ARCH)
    assert os.path.exists(build.LIB)


def test_argument_errors_without_device(fundem):
    import ctypes as C
    L = fundem.lib()
    assert L.fundem_create(None, 0, None) == 1  # FUNDEM_ERR_ARG
    h = C.c_void_p()
    r = L.fundem_create(C.byref(h), 10_000, None)
    assert r == 2  # no such device: FUNDEM_ERR_CUDA, never a crash


def test_mass_properties_host_matches_oracle(fundem, oracle_mod):
    """The library's host mass-property routine follows the same loop order
    as the reference (LSSolver.h:503-565): bitwise equal to the oracle."""
    import numpy as np
    from fundem_b200 import scenario as S
    g = S.superellipsoid_template(1e-3, 0.9e-3, 1.1e-3, 0.5, 1.0, n=20)
    a = fundem.mass_properties(2500.0, g.origin, g.spacing, g.size, g.sdf)
    b = oracle_mod.mass_properties(2500.0, g.origin, g.spacing, g.size, g.sdf)
    assert a[0] == b[0]
    assert np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])


@pytest.mark.parametrize("lang", ["c", "c++"])
def test_header_is_plain_c(tmp_path, lang):
    """include/fundem_b200.h compiles on its own as C99 and as C++17: plain
    types, extern "C" linkage, no library types in the signatures."""
    import shutil
    import subprocess
    cc = shutil.which("gcc" if lang == "c" else "g++")
    if cc is None:
        pytest.skip("no host compiler")
    src = tmp_path / ("probe.c" if lang == "c" else "probe.cpp")
    src.write_text('#include "fundem_b200.h"\nint probe(void) { return FUNDEM_OK + FUNDEM_INERTIA_PHYSICAL; }\n')
    std = "-std=c99" if lang == "c" else "-std=c++17"
    subprocess.check_call([cc, std, "-Wall", "-Werror", "-pedantic", "-fsyntax-only", "-I",
                           os.path.join(ROOT, "include"), str(src)])


def test_null_simulation_is_an_argument_error(fundem):
    L = fundem.lib()
    assert L.fundem_set_inertia_mode(None, 0) == 1
    assert L.fundem_set_periodic_sector(None, 1) == 1
    assert L.fundem_set_precision(None, 0) == 1
    assert L.fundem_adjoint_begin(None, 10) == 1
