import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TESTS = os.path.dirname(os.path.abspath(__file__))
for p in (ROOT, TESTS):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(TESTS, "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def fundem():
    import fundem_b200 as F
    from fundem_b200 import build
    build.build()
    F.lib()
    return F


def load_golden(name):
    path = os.path.join(GOLDEN, f"{name}.npz")
    if not os.path.exists(path):
        pytest.skip(f"golden fixture {name}.npz not generated")
    return dict(np.load(path, allow_pickle=False))


def canonical(c):
    """Contact list sorted by (node, partner)."""
    o = np.lexsort((c["slave"], c["master"]))
    return {k: (v[o] if hasattr(v, "__len__") and len(v) == len(o) else v) for k, v in c.items()}


def keys(c):
    return np.stack([np.asarray(c["master"], np.int64), np.asarray(c["slave"], np.int64)], axis=1)


def golden_contacts(g, step, kind):
    p = f"s{step}_{kind}_"
    return {k[len(p):]: v for k, v in g.items() if k.startswith(p)}


def golden_state(g, step):
    p = f"s{step}_"
    return {k: g[p + k] for k in ("pos", "vel", "angvel", "quat", "force", "torque")}


def rel_err(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    scale = max(np.abs(b).max(initial=0.0), 1e-300)
    return float(np.abs(a - b).max(initial=0.0) / scale)


_SHA = {}


def scenario_sha(name):
    """SHA-256 of the reference-driver file for a parity case, rebuilt here."""
    if name not in _SHA:
        import hashlib
        import tempfile
        import parity_cases as PC
        from oracle import scenario_io as SIO
        sc = PC.CASES[name]()
        n, dumps = PC.REF_STEPS[name]
        with tempfile.TemporaryDirectory() as d:
            path = os.path.join(d, "s.bin")
            SIO.write_reference_scenario(sc, path, n, dumps)
            with open(path, "rb") as f:
                _SHA[name] = hashlib.sha256(f.read()).hexdigest()
    return _SHA[name]
