"""The cell-hash sort (fundem_hash_sort, the library's replacement for the
sort of buildHashStartEnd) and the two cell-table forms on the GPU.

* The permutation equals numpy's stable argsort bit for bit (hashes outside
  [0, num_cells) last), for grids below and above 2^31 cells, with repeated
  keys, and for 0, 1 and 4097 objects.
* A simulation whose grid has more cells than a dense table should hold
  (the cluster case in a domain of several metres) keeps a hash table of its
  occupied cells: its detection and steps match the oracle, which hashes into
  the reference's dense grid, bit for bit at the first detection.
"""
import numpy as np
import pytest
import torch

from conftest import canonical, keys, rel_err
import parity_cases as PC

pytestmark = pytest.mark.gpu


def _sort(fundem, h, num):
    d = torch.tensor(h, dtype=torch.int64, device="cuda")
    out = torch.empty(len(h), dtype=torch.int32, device="cuda")
    sh = torch.empty(len(h), dtype=torch.int64, device="cuda")
    if len(h):
        fundem.hash_sort(d.data_ptr(), len(h), num, out.data_ptr(), sh.data_ptr())
    torch.cuda.synchronize()
    return out.cpu().numpy(), sh.cpu().numpy()


def _want(h, num):
    k = np.where((h >= 0) & (h < num), h, np.iinfo(np.int64).max)
    order = np.argsort(k, kind="stable").astype(np.int32)
    sk = h[order].copy()
    sk[(sk < 0) | (sk >= num)] = -1
    return order, sk


@pytest.mark.parametrize("num,n,dup", [(255, 4097, False), (256, 100000, True), (65536 * 3, 262144, True),
                                       (5_000_000_000, 200000, False), ((1 << 40) + 7, 50000, True),
                                       (1, 1000, True), (1000, 1, False)])
def test_sort_equals_numpy_stable_argsort(fundem, num, n, dup):
    rng = np.random.default_rng(n + num % 1000)
    hi = max(num // 16, 1) if dup else num
    h = rng.integers(0, hi, n, dtype=np.int64)
    h[rng.random(n) < 0.05] = -1            # objects outside the grid
    if n > 10:
        h[3] = num                          # a hash past the last cell counts as outside too
    order, sk = _sort(fundem, h, num)
    want, wsk = _want(h, num)
    assert np.array_equal(order, want)
    assert np.array_equal(sk, wsk)


def test_sort_empty(fundem):
    order, _ = _sort(fundem, np.zeros(0, np.int64), 100)
    assert order.size == 0


def test_hashed_cell_table_matches_oracle(fundem, oracle_mod):
    sc = PC.cluster()
    sc.domain_max = sc.domain_min + np.array([6.0, 6.0, 6.0])   # far more cells than a dense table keeps
    g = fundem.Simulation.from_scenario(sc)
    grid = g.grid()
    assert int(np.prod(grid["size"].astype(np.int64))) > (1 << 22)
    o = oracle_mod.OracleWorld.from_scenario(sc)
    g.detect()
    o.initial_detect()
    for k in range(2):
        a, b = canonical(g.contacts(k)), canonical(o.contacts(k))
        assert np.array_equal(keys(a), keys(b))
        assert np.array_equal(a["overlap"], b["overlap"])
    for s in range(8):
        g.step(1)
        o.step(1)
        for k in range(2):
            assert np.array_equal(keys(canonical(g.contacts(k))), keys(canonical(o.contacts(k)))), (s, k)
        assert rel_err(g.state()["force"], o.state()["force"]) < 1e-10
    g.sync()
