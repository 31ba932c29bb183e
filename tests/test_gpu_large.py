"""Inputs above 2^30 keys: each pass runs as several launches ("portions" of
at most 2^30 keys, the look-back's 30-bit counts) with per-digit counts
carried between them, and above 2^31 keys with 64-bit offsets. Keys are made
and checked on the device (sorted in radix order, same multiset: sum and sum
of squares, both wrapping in 64 bits)."""
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ts():
    import turbosort_b200 as ts

    return ts


def _multiset(v64):
    return int(v64.sum().item()), int((v64 * v64).sum().item())


@pytest.mark.parametrize("n, t", [((1 << 30) + 12345, "u32"), ((1 << 31) + 777, "u32"), ((1 << 30) + 99, "u64")],
                         ids=["u32-two-portions", "u32-three-portions-64bit-offsets", "u64-two-portions"])
def test_sorts_above_one_portion(ts, n, t):
    import torch

    g = torch.Generator(device="cuda")
    g.manual_seed(n)
    if t == "u32":
        x = torch.randint(-2**31, 2**31, (n,), dtype=torch.int32, device="cuda", generator=g)
        before = _multiset(x.to(torch.int64) & 0xFFFFFFFF)
        ts.sort(x.view(torch.uint32))
        torch.cuda.synchronize()
        y = x ^ torch.tensor(-2**31, dtype=torch.int32, device="cuda")  # unsigned order as signed
        assert bool((y[1:] >= y[:-1]).all().item())
        del y
        assert _multiset(x.to(torch.int64) & 0xFFFFFFFF) == before
    else:
        x = torch.randint(-2**62, 2**62, (n,), dtype=torch.int64, device="cuda", generator=g)
        before = _multiset(x)
        ts.sort(x.view(torch.uint64))
        torch.cuda.synchronize()
        y = x ^ torch.tensor(-2**63, dtype=torch.int64, device="cuda")
        assert bool((y[1:] >= y[:-1]).all().item())
        del y
        assert _multiset(x) == before
    del x
    torch.cuda.empty_cache()
