"""Parity of the host-slice sort with its copies overlapped (chunked copies
in, chunk sorts, pairwise device merges, sliced copies out) with the oracle,
through the C ABI. Every comparison is bit-exact; the pipeline is forced on
at small sizes by setting its size threshold to zero.
"""
import zlib

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

PIPE_TYPES = [t for t in O.TYPES if t not in ("u8", "i8")]


@pytest.fixture(scope="module")
def ts():
    import turbosort_b200 as ts

    return ts


def gen(t, n, shape, rng):
    kd = O.KEY_DTYPE[t]
    b = rng.integers(0, 2**64, size=n, dtype=np.uint64)
    if shape == "few":
        b %= np.uint64(7)
    elif shape == "const":
        b[:] = b[0]
    a = b.astype(kd).view(O.NP_DTYPE[t])
    if shape == "asc":
        a = O.sort(a)
    elif shape == "desc":
        a = O.sort(a)[::-1].copy()
    if t in ("f32", "f64") and shape == "random":
        ft = np.float32 if t == "f32" else np.float64
        sp = np.array([np.nan, -np.nan, np.inf, -np.inf, 0.0, -0.0], dtype=ft)
        idx = rng.integers(0, n, size=max(1, n // 50))
        a[idx] = sp[rng.integers(0, sp.size, size=idx.size)]
    return a


def run(ts, ctx, a):
    got = a.copy()
    ts.sort(got, ctx)
    return got


@pytest.mark.parametrize("t", PIPE_TYPES)
def test_pipeline_matches_oracle(ts, t):
    ctx = ts.Context(0)
    rng = np.random.default_rng(zlib.crc32(b"pipe " + t.encode()))
    for chunks in (2, 8, 64):
        ctx.transfer_pipeline(chunks, 0)
        for n in (chunks * 256, chunks * 256 + 1, 100_003, (1 << 20) + 17):
            for shape in ("random", "few", "asc", "desc", "const"):
                a = gen(t, n, shape, rng)
                got = run(ts, ctx, a)
                assert got.tobytes() == O.sort(a).tobytes(), (t, chunks, n, shape)
    ctx.close()


def test_pipeline_runs_merges_and_agrees_with_serial(ts):
    ctx = ts.Context(0)
    rng = np.random.default_rng(3)
    a = gen("u32", 3_000_001, "random", rng)
    ctx.transfer_pipeline(1, 0)
    serial = run(ts, ctx, a)
    ctx.transfer_pipeline(8, 0)
    ctx.reset_timings()
    ctx.enable_timing(True)
    before = ts.lib().ts_ctx_launches(ctx.handle)
    piped = run(ts, ctx, a)
    ctx.enable_timing(False)
    assert "merge" in ctx.timings()
    # 8 chunk sorts, 7 merges: each merge is a split launch plus tile launches
    assert ts.lib().ts_ctx_launches(ctx.handle) - before >= 8 + 14
    assert piped.tobytes() == serial.tobytes() == O.sort(a).tobytes()
    ctx.close()


def test_default_threshold_and_repeated_calls(ts):
    """2^24 u32 keys (64 MiB) reach the default threshold; repeated and
    differently sized calls on one context reuse and grow its buffers."""
    ctx = ts.Context(0)
    rng = np.random.default_rng(5)
    for n in (1 << 24, 1 << 24, (1 << 22) + 3, (1 << 24) + 4097):
        a = gen("u32", n, "random", rng)
        ctx.transfer_pipeline(8, 0 if n < (1 << 24) else 64 << 20)
        assert run(ts, ctx, a).tobytes() == O.sort(a).tobytes(), n
    ctx.close()


def test_pinned_host_slice(ts):
    import torch

    ctx = ts.Context(0)
    ctx.transfer_pipeline(16, 0)
    rng = np.random.default_rng(9)
    for t, n in (("f32", 2_000_003), ("i64", 1_000_033)):
        a = gen(t, n, "random", rng)
        pinned = torch.empty(a.nbytes, dtype=torch.uint8, pin_memory=True).numpy().view(a.dtype)
        np.copyto(pinned, a)
        ts.sort(pinned, ctx)
        assert pinned.tobytes() == O.sort(a).tobytes(), t
    ctx.close()


def test_pageable_slice_larger_than_the_staging_ring(ts):
    """A pageable slice goes through four pinned 32 MiB slots; 512 MiB of u64
    keys in two chunks wraps the ring several times each way."""
    ctx = ts.Context(0)
    ctx.transfer_pipeline(2, 0)
    rng = np.random.default_rng(11)
    a = gen("u64", (1 << 26) + 12345, "random", rng)
    got = run(ts, ctx, a)
    assert got.tobytes() == O.sort(a).tobytes()
    ctx.close()


@pytest.mark.parametrize("t", PIPE_TYPES)
def test_keys_order_pipeline_matches_oracle(ts, t):
    """sort_by_key's order() through the pipeline: chunk orders merged by the
    keys they point to. Few distinct keys make every merge decide ties, where
    only a stable merge gives the crate's permutation."""
    ctx = ts.Context(0)
    rng = np.random.default_rng(zlib.crc32(b"order " + t.encode()))
    for chunks in (2, 8):
        ctx.transfer_pipeline(chunks, 0)
        for n in (chunks * 256, chunks * 256 + 1, 100_003, (1 << 20) + 17):
            for shape in ("random", "few", "asc", "desc", "const"):
                a = gen(t, n, shape, rng)
                got = ts.keys_order(a, ctx)
                assert got.tobytes() == O.sort_by_key_order(a).tobytes(), (t, chunks, n, shape)
    ctx.close()


def test_keys_order_pipeline_pinned_and_large(ts):
    """Pinned keys and order (straight DMAs), and a pageable 2^25-key u64
    slice whose keys and order wrap the staging ring."""
    import torch

    ctx = ts.Context(0)
    rng = np.random.default_rng(13)
    ctx.transfer_pipeline(16, 0)
    a = gen("f64", 3_000_017, "few", rng)
    keys = torch.empty(a.nbytes, dtype=torch.uint8, pin_memory=True).numpy().view(a.dtype)
    np.copyto(keys, a)
    out = torch.empty(a.size * 4, dtype=torch.uint8, pin_memory=True).numpy().view(np.uint32)
    ts.keys_order(keys, ctx, out=out)
    assert out.tobytes() == O.sort_by_key_order(a).tobytes()
    ctx.transfer_pipeline(8, 64 << 20)
    b = gen("u64", (1 << 25) + 999, "random", rng) % np.uint64(1 << 20)
    assert ts.keys_order(b, ctx).tobytes() == O.sort_by_key_order(b).tobytes()
    ctx.close()


def test_apply_order_pipeline_matches_oracle(ts):
    """Host apply_order with the copies overlapped (the gather in output
    slices, each copied back while the next is gathered), for element sizes
    that take every gather word width, pageable and pinned."""
    import torch

    ctx = ts.Context(0)
    ctx.transfer_pipeline(8, 0)
    rng = np.random.default_rng(17)
    for n in (8 * 256, 100_003, (1 << 20) + 5):
        order = rng.permutation(n).astype(np.uint32)
        for elem in (1, 3, 4, 8, 12, 16, 24):
            data = rng.integers(0, 256, size=(n, elem), dtype=np.uint8)
            want = O.apply_order(data, order)
            got = data.copy()
            ts.apply_order(got, order, ctx)
            assert got.tobytes() == want.tobytes(), (n, elem)
        pinned = torch.empty(n * 16, dtype=torch.uint8, pin_memory=True).numpy().reshape(n, 16)
        data = rng.integers(0, 256, size=(n, 16), dtype=np.uint8)
        np.copyto(pinned, data)
        ts.apply_order(pinned, order, ctx)
        assert pinned.tobytes() == O.apply_order(data, order).tobytes(), n
    ctx.close()


def _segments_case(rng, t, count, huge):
    lengths = rng.integers(0, 3000, size=count)
    lengths[rng.integers(0, count, size=count // 10)] = 0
    if huge:
        lengths[count // 3] = (1 << 22) + 5  # above the host path's limit: the device-wide sort
    offs = np.zeros(count + 1, dtype=np.uint64)
    offs[1:] = np.cumsum(lengths) + 77  # keys before the first segment and after the last stay put
    offs[0] = 77
    n = int(offs[-1]) + 123
    return gen(t, n, "random", rng), offs


def _segments_want(a, offs):
    want = a.copy()
    for i in range(offs.size - 1):
        lo, hi = int(offs[i]), int(offs[i + 1])
        if hi - lo > 1:
            want[lo:hi] = O.sort(a[lo:hi])
    return want


@pytest.mark.parametrize("t", ["u32", "f32", "u64", "i16"])
def test_segments_pipeline_matches_oracle(ts, t):
    """Host segmented sort in groups of whole segments, each sorted while
    later groups cross and copied back at once (pinned) or after (pageable)."""
    import torch

    ctx = ts.Context(0)
    rng = np.random.default_rng(zlib.crc32(b"seg " + t.encode()))
    for chunks, count, huge in ((2, 50, False), (8, 1500, True), (64, 700, False)):
        ctx.transfer_pipeline(chunks, 0)
        a, offs = _segments_case(rng, t, count, huge)
        want = _segments_want(a, offs)
        got = a.copy()
        ts.sort_segments(got, offs, ctx)
        assert got.tobytes() == want.tobytes(), (t, chunks, count)
        pinned = torch.empty(a.nbytes, dtype=torch.uint8, pin_memory=True).numpy().view(a.dtype)
        np.copyto(pinned, a)
        ts.sort_segments(pinned, offs, ctx)
        assert pinned.tobytes() == want.tobytes(), (t, chunks, count, "pinned")
    ctx.close()


def test_learned_sort_of_a_pageable_slice(ts):
    """The learned sort needs every key before it partitions, so its host
    copies do not overlap it; a pageable slice crosses through the staging
    slots (here larger than the ring) and comes back sorted."""
    from turbosort_b200 import workloads as W

    ctx = ts.Context(0)
    ctx.transfer_pipeline(8, 0)
    for a in (W.lognormal_f64((1 << 24) + 3), W.gauss_mix_u64(1 << 21)):
        got = a.copy()
        ts.sort_learned(got, ctx=ctx)
        assert got.tobytes() == O.sort(a).tobytes(), a.dtype
    ctx.close()


def test_rejects_bad_chunk_counts(ts):
    ctx = ts.Context(0)
    for bad in (0, 3, 12, 128):
        with pytest.raises(ts.TurbosortError):
            ctx.transfer_pipeline(bad, 0)
    ctx.close()
