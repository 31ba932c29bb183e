"""More input shapes from the crate's own tests, on the device, bit-exact
against the oracle.

- the 0-1 principle for the small-slice networks (the crate checks its NEON
  networks on every 0/1 input up to 16 keys, src/arch/aarch64/neon.rs:227-253):
  every 0/1 slice up to 12 keys through the single-slice sort, and every 0/1
  segment of 16 keys (plus random 0/1 segments of every on-chip length bin)
  through the segmented sort;
- the structured shapes of tests/correctness.rs:128-245 (split top bit,
  correlated top bytes, 1000 distinct values, heavy tail, pipe organ, equal
  buckets) at tier and tile boundaries, for every key width.
"""
import zlib

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ts():
    import turbosort_b200 as ts

    return ts


def test_zero_one_principle_single_slices(ts):
    for n in range(2, 13):
        codes = np.arange(1 << n, dtype=np.uint32)
        bits = ((codes[:, None] >> np.arange(n, dtype=np.uint32)) & 1).astype(np.uint32)
        for row in bits:
            got = row.copy()
            ts.sort(got)
            ones = int(row.sum())
            assert got.tolist() == [0] * (n - ones) + [1] * ones, row.tolist()


def test_zero_one_principle_segments(ts):
    # every 0/1 segment of 16 keys (one warp each), then random 0/1 segments
    # of lengths across the on-chip bins (33 .. 16384)
    codes = np.arange(1 << 16, dtype=np.uint32)
    keys = ((codes[:, None] >> np.arange(16, dtype=np.uint32)) & 1).astype(np.uint16).reshape(-1)
    offs = np.arange(0, keys.size + 1, 16, dtype=np.uint64)
    got = keys.copy()
    ts.sort_segments(got, offs)
    want = np.sort(keys.reshape(-1, 16), axis=1).reshape(-1)
    assert got.tobytes() == want.tobytes()
    rng = np.random.default_rng(21)
    lengths = np.concatenate([rng.integers(33, 257, 300), rng.integers(257, 4097, 100),
                              rng.integers(4097, 16385, 20)])
    offs = np.zeros(lengths.size + 1, dtype=np.uint64)
    offs[1:] = np.cumsum(lengths)
    keys = rng.integers(0, 2, size=int(offs[-1])).astype(np.uint32)
    got = keys.copy()
    ts.sort_segments(got, offs)
    for i in range(lengths.size):
        lo, hi = int(offs[i]), int(offs[i + 1])
        assert got[lo:hi].tobytes() == np.sort(keys[lo:hi]).tobytes(), i


def structured(t, n, shape, rng):
    """Keys of type t with the shape's radix-key pattern (as the crate's
    u64 shapes, cut to the key width)."""
    kd = O.KEY_DTYPE[t]
    w = np.dtype(kd).itemsize * 8
    top = np.uint64(w - 1)
    r = rng.integers(0, 2**64, size=n, dtype=np.uint64)
    if shape == "split_top_bit":
        b = (r >> np.uint64(64 - w + 1)) | (rng.integers(0, 2, size=n, dtype=np.uint64) << top)
    elif shape == "correlated_top":
        low = r & np.uint64(0xFF)
        b = (low << np.uint64(w - 8)) | (r & np.uint64(0xFF)) if w > 8 else low
    elif shape == "distinct_1000":
        pool = rng.integers(0, 2**64, size=1000, dtype=np.uint64)
        b = pool[rng.integers(0, 1000, size=n)]
    elif shape == "heavy_tail":
        b = np.where(rng.random(n) < 0.99, r & np.uint64(0xFF), r)
    elif shape == "pipe_organ":
        half = np.sort(r[: (n + 1) // 2] >> np.uint64(64 - w))
        b = np.concatenate([half, half[: n // 2][::-1]])
    elif shape == "equal_buckets":
        # every 8-bit digit value equally often in every byte
        b = np.zeros(n, dtype=np.uint64)
        for byte in range(w // 8):
            b |= rng.permutation(np.arange(n, dtype=np.uint64) % np.uint64(256)) << np.uint64(8 * byte)
    else:
        raise ValueError(shape)
    return (b & np.uint64((1 << w) - 1 if w < 64 else 2**64 - 1)).astype(kd).view(O.NP_DTYPE[t])


SHAPES = ["split_top_bit", "correlated_top", "distinct_1000", "heavy_tail", "pipe_organ", "equal_buckets"]


@pytest.mark.parametrize("t", ["u16", "u32", "i32", "f32", "u64", "i64", "f64"])
def test_structured_shapes(ts, t):
    rng = np.random.default_rng(zlib.crc32(b"shapes " + t.encode()))
    for n in (4095, 4097, 11264, 11265, 65537, 300_001):
        for shape in SHAPES:
            a = structured(t, n, shape, rng)
            got = a.copy()
            ts.sort(got)
            assert got.tobytes() == O.sort(a).tobytes(), (t, n, shape)
            order = ts.keys_order(a)
            assert order.tobytes() == O.sort_by_key_order(a).tobytes(), (t, n, shape, "order")


def adversarial(t, n, shape, rng):
    """Patterns aimed at radix sorts (the crate's adversarial cases,
    tests/correctness.rs:575-635): digit-aligned sawtooth, alternating
    extremes, one outlier, keys differing in one byte only."""
    kd = O.KEY_DTYPE[t]
    w = np.dtype(kd).itemsize * 8
    i = np.arange(n, dtype=np.uint64)
    full = np.uint64((1 << w) - 1 if w < 64 else 2**64 - 1)
    if shape == "sawtooth_256":
        b = i % np.uint64(256)
    elif shape == "sawtooth_65536":
        b = i % np.uint64(65536)
    elif shape == "alternating_extremes":
        b = np.where(i % np.uint64(2) == 0, np.uint64(0), full)
    elif shape == "one_outlier":
        b = np.full(n, 7, dtype=np.uint64)
        b[n // 2] = full
    elif shape == "top_byte_only":
        b = rng.integers(0, 256, size=n, dtype=np.uint64) << np.uint64(w - 8)
    elif shape == "bottom_byte_only":
        b = rng.integers(0, 256, size=n, dtype=np.uint64) | (full & ~np.uint64(0xFF))
    else:
        raise ValueError(shape)
    return (b & full).astype(kd).view(O.NP_DTYPE[t])


ADVERSARIAL = ["sawtooth_256", "sawtooth_65536", "alternating_extremes", "one_outlier", "top_byte_only",
               "bottom_byte_only"]


@pytest.mark.parametrize("t", ["u16", "u32", "i32", "f32", "u64", "f64"])
def test_adversarial_shapes(ts, t):
    rng = np.random.default_rng(zlib.crc32(b"adv " + t.encode()))
    for n in (4096, 4097, 65536, 300_000):
        for shape in ADVERSARIAL:
            a = adversarial(t, n, shape, rng)
            got = a.copy()
            ts.sort(got)
            assert got.tobytes() == O.sort(a).tobytes(), (t, n, shape)
            order = ts.keys_order(a)
            assert order.tobytes() == O.sort_by_key_order(a).tobytes(), (t, n, shape, "order")
