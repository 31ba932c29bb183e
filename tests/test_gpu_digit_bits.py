"""The plain LSD at every digit width from 4 to 11 bits.

The crate sorts with 8-bit digits and long u64 slices with 11-bit ones
(src/radix/mod.rs:43-54, :518-600); here the width is set per key width and
length bin (ts_lsd_digit_bits). Each width sorts bit-exactly like the oracle
for every key transform (unsigned, signed, IEEE float with NaN of both signs,
+-0 and +-inf), at a length just above the small tier, at a ragged length of
several tiles and at one of many tiles (a long look-back chain); the plan the
device chose is read back: one pass per varying digit of that width,
none for presorted input, a reversal for descending input."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KINDS = [np.uint16, np.int16, np.uint32, np.int32, np.float32, np.uint64, np.int64, np.float64]
BITS = [4, 5, 6, 7, 9, 10, 11]


@pytest.fixture(scope="module")
def env():
    import torch

    import turbosort_b200 as ts
    from oracle import oracle as O

    ctx = ts.Context(0)
    return torch, ts, O, ctx


def _keys(t, n, seed):
    rng = np.random.default_rng(seed)
    w = rng.integers(0, 2**63, size=n, dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, size=n, dtype=np.uint64)
    a = w.astype({2: np.uint16, 4: np.uint32, 8: np.uint64}[np.dtype(t).itemsize]).view(t).copy()
    if np.dtype(t).kind == "f":
        a[::97] = np.nan
        a[1::97] = -np.nan
        a[2::101] = 0.0
        a[3::101] = -0.0
        a[4::103] = np.inf
        a[5::103] = -np.inf
    return a


def _sort(env, a, bits):
    """Sort a device copy of `a` with `bits`-bit digits; the output and the plan."""
    torch, ts, O, ctx = env
    w = a.dtype.itemsize
    ctx.lsd_digit_bits(w, [bits] * 3)
    try:
        iview = {2: np.int16, 4: np.int32, 8: np.int64}[w]
        tdt = {"u": {2: torch.uint16, 4: torch.uint32, 8: torch.uint64},
               "i": {2: torch.int16, 4: torch.int32, 8: torch.int64},
               "f": {4: torch.float32, 8: torch.float64}}[a.dtype.kind][w]
        d = torch.from_numpy(a.view(iview).copy()).cuda()
        ts.sort(d.view(tdt), ctx)
        ctx.synchronize()
        info = ctx.last_sort_info()
        return d.cpu().numpy().view(a.dtype), info
    finally:
        ctx.lsd_digit_bits(w, [8, 8, 8])


def _digits(width_bits, bits):
    return -(-width_bits // bits)


@pytest.mark.parametrize("bits", BITS)
@pytest.mark.parametrize("t", KINDS)
def test_every_width_matches_the_oracle(env, t, bits):
    _, _, O, _ = env
    W = 8 * np.dtype(t).itemsize
    for i, n in enumerate([4_097, 70_001, 1_000_003]):
        a = _keys(t, n, 100 * bits + 7 * i + np.dtype(t).itemsize)
        got, info = _sort(env, a, bits)
        assert got.tobytes() == O.sort(a).tobytes(), f"{np.dtype(t)} n={n} bits={bits}"
        assert info["tier"] == 3 and info["digit_bits"] == bits and info["divert_shift"] == 0, info
        # random full-width keys vary in every digit
        assert info["passes"] == _digits(W, bits), info
        assert info["pass_digit"] == list(range(_digits(W, bits))), info


@pytest.mark.parametrize("bits", [9, 10, 11])
@pytest.mark.parametrize("t", [np.uint32, np.float32, np.uint64, np.int64])
def test_many_tiles(env, t, bits):
    """(2^22 + 5) keys: hundreds of tiles per pass at every wide width."""
    _, _, O, _ = env
    a = _keys(t, (1 << 22) + 5, 7 * bits)
    got, info = _sort(env, a, bits)
    assert got.tobytes() == O.sort_parallel(a).tobytes()
    assert info["digit_bits"] == bits


@pytest.mark.parametrize("bits", BITS + [8])
def test_plan_shapes(env, bits):
    """Narrow ranges take one pass per varying digit of the width; presorted
    input takes none; descending input is reversed; few distinct keys."""
    _, _, O, _ = env
    rng = np.random.default_rng(bits)
    n = 200_003
    # 20 varying low bits of u32 keys
    a = rng.integers(0, 1 << 20, size=n, dtype=np.uint32)
    got, info = _sort(env, a, bits)
    assert got.tobytes() == O.sort(a).tobytes()
    assert info["passes"] == _digits(20, bits), info
    # varying bits only in the top 12 of u64 keys (the low digits are constant)
    b = rng.integers(0, 1 << 12, size=n, dtype=np.uint64) << np.uint64(52)
    got, info = _sort(env, b, bits)
    assert got.tobytes() == O.sort(b).tobytes()
    assert info["passes"] == _digits(64, bits) - 52 // bits, info
    s = np.sort(a)
    got, info = _sort(env, s, bits)
    assert got.tobytes() == s.tobytes() and info["passes"] == 0, info
    got, info = _sort(env, s[::-1].copy(), bits)
    assert got.tobytes() == s.tobytes() and info["passes"] == 0 and info["mode"] == 2, info
    c = rng.integers(0, 3, size=n, dtype=np.uint64) * np.uint64(0x0123456789ABCDEF)
    got, _ = _sort(env, c, bits)
    assert got.tobytes() == O.sort(c).tobytes()


def test_host_slices_and_rejected_widths(env):
    """The width applies to host slices too; widths outside 4..11 are refused."""
    torch, ts, O, ctx = env
    a = _keys(np.float64, 300_001, 3)
    ctx.lsd_digit_bits(8, [11, 11, 11])
    try:
        got = a.copy()
        ts.sort(got, ctx)
        assert got.tobytes() == O.sort(a).tobytes()
        assert ctx.last_sort_info()["digit_bits"] == 11
    finally:
        ctx.lsd_digit_bits(8, [8, 8, 8])
    for bad in ([3, 8, 8], [8, 12, 8]):
        with pytest.raises(ts.TurbosortError):
            ctx.lsd_digit_bits(4, bad)
    assert ctx.lsd_digit_bits(4) == [8, 8, 8]
