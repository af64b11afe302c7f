"""The prefix-sum entry point (the reference's buildPrefixSum) against
torch.cumsum, including tile-boundary sizes and empty input."""
import pytest

pytestmark = pytest.mark.gpu

SIZES = [0, 1, 7, 4095, 4096, 4097, 12345, 4096 * 4096 + 3, 5_000_000]


@pytest.mark.parametrize("n", SIZES)
def test_prefix_sum_matches_cumsum(fundem, n):
    import torch
    g = torch.Generator(device="cuda").manual_seed(n)
    x = torch.randint(0, 9, (n,), device="cuda", dtype=torch.int32, generator=g)
    y = fundem.prefix_sum(x)
    torch.cuda.synchronize()
    if n:
        ref = torch.cumsum(x.to(torch.int64), 0).to(torch.int32)
        assert torch.equal(y, ref)
