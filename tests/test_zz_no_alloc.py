"""The allocation-free prefix sum (fundem_prefix_sum_noalloc) against the
allocating one (fundem_prefix_sum), both called through the C ABI.

Some callers of this library cannot allocate device memory when they need a
scan (a memory budget already reserved by another allocator, or no tolerance
for cudaMalloc's implicit synchronisation); for them the scratch lives in a
fixed device array of the library.  This file runs last so that a failure
here does not stop the other tests; it passes on its own in a fresh process
as well.  Integer results, so the comparison is exact."""
import ctypes as C

import pytest

pytestmark = pytest.mark.gpu

MAX = 16777216  # FUNDEM_NOALLOC_SCAN_MAX in include/fundem_b200.h


def _scan(L, fn, x):
    import torch
    y = torch.full_like(x, -7)
    r = getattr(L, fn)(C.c_void_p(y.data_ptr()), C.c_void_p(x.data_ptr()), C.c_longlong(x.numel()), None)
    return r, y


@pytest.mark.parametrize("n", [1, 4095, 4096, 4097, 123457, 3_000_001, MAX])
def test_noalloc_prefix_sum_matches_allocating_entry_point(fundem, n):
    import torch
    L = fundem.lib()
    g = torch.Generator(device="cuda").manual_seed(1234 + n)
    for call in range(2):  # two calls in a row share the scratch array
        x = torch.randint(0, 5, (n,), device="cuda", dtype=torch.int32, generator=g)
        r1, ref = _scan(L, "fundem_prefix_sum", x)
        r2, got = _scan(L, "fundem_prefix_sum_noalloc", x)
        torch.cuda.synchronize()
        assert r1 == 0 and r2 == 0
        assert torch.equal(got, ref), (n, call)
        assert int(got[-1]) == int(x.to(torch.int64).sum())


def test_noalloc_prefix_sum_rejects_sizes_beyond_the_limit(fundem):
    L = fundem.lib()
    assert L.fundem_prefix_sum_noalloc(C.c_void_p(1), C.c_void_p(1), C.c_longlong(MAX + 1), None) == 1
    assert L.fundem_prefix_sum_noalloc(None, None, C.c_longlong(0), None) == 0
