"""The segmented batch sort: every segment must equal the oracle's sort of
that slice (the crate's sort per slice, as in its small_batches benchmark),
for all ten types, across every length bin boundary, with each method."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

EDGES = [0, 1, 2, 3, 31, 32, 33, 100, 255, 256, 257, 1000, 1024, 1025, 4095, 4096, 4097, 8191, 8192, 8193,
         16383, 16384, 16385, 40000, 65536]


@pytest.fixture(scope="module")
def ts():
    import turbosort_b200 as ts

    return ts


def batch(t, lengths, rng, shape="random"):
    offs = np.zeros(len(lengths) + 1, dtype=np.uint64)
    offs[1:] = np.cumsum(lengths)
    n = int(offs[-1])
    b = rng.integers(0, 2**64, size=n, dtype=np.uint64)
    if shape == "few":
        b %= np.uint64(7)
    elif shape == "range16":
        b &= np.uint64(0xFFFF)
    return b.astype(O.KEY_DTYPE[t]).view(O.NP_DTYPE[t]), offs


def expected(a, offs):
    out = a.copy()
    for i in range(len(offs) - 1):
        lo, hi = int(offs[i]), int(offs[i + 1])
        if hi - lo > 1:
            out[lo:hi] = O.sort(a[lo:hi])
    return out


@pytest.mark.parametrize("t", O.TYPES)
def test_segments_match_oracle(ts, t):
    rng = np.random.default_rng(21)
    lengths = EDGES + list(rng.integers(0, 3000, size=200))
    for shape in ("random", "few", "range16"):
        a, offs = batch(t, lengths, rng, shape)
        want = expected(a, offs)
        got = a.copy()
        ts.sort_segments(got, offs)
        assert got.tobytes() == want.tobytes(), (t, shape)


@pytest.mark.parametrize("t", ["u32", "f32", "u64", "i16", "i64", "f64"])
@pytest.mark.parametrize("method", [0, 1, 2, 3, 4, 5, 6])
def test_each_method(ts, t, method):
    """Every method in every block bin it serves: the warp-per-segment
    methods in the first bin (4) and, for keys of up to 4 bytes, the second
    (5); the grouped MSD method (6) in the third and fourth, for keys of 4 and
    8 bytes. Bins a method does not serve take the MSD method meanwhile."""
    ctx = ts.Context(0)
    w = np.dtype(O.NP_DTYPE[t]).itemsize
    if method == 5 and w > 4:
        pytest.skip("the 32-keys-a-lane warp method takes keys of up to 4 bytes")
    if method == 6 and w < 4:
        pytest.skip("the grouped MSD method takes keys of 4 and 8 bytes")
    ts.segments_methods(w, ctx, {4: [4, 3, 3, 3], 5: [4, 5, 3, 3], 6: [4, 3, 6, 6]}.get(method, [method] * 4))
    rng = np.random.default_rng(method)
    lengths = list(rng.integers(33, 16384 if w < 8 else 8192, size=60)) + [33, 256, 257, 1024, 1025, 4096, 4097]
    a, offs = batch(t, lengths, rng)
    got = a.copy()
    ts.sort_segments(got, offs, ctx)
    assert got.tobytes() == expected(a, offs).tobytes()


def test_device_segments_and_graph_replay(ts):
    import torch

    ctx = ts.Context(0)
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    rng = np.random.default_rng(5)
    lengths = [int(x) for x in np.floor(np.exp(rng.random(3000) * np.log(65536))).astype(np.int64)]
    a, offs = batch("f32", lengths, rng)
    want = expected(a, offs)
    d_off = torch.from_numpy(offs.view(np.int64)).cuda()
    master = torch.from_numpy(a.view(np.int32)).cuda()
    lib = ts.lib()
    d = torch.empty_like(master)
    for _ in range(3):  # the second and third calls replay the captured graph
        d.copy_(master)
        before = lib.ts_ctx_launches(ctx.handle)
        ts.sort_segments(d.view(torch.float32), d_off, ctx)
        ctx.synchronize()
        assert lib.ts_ctx_launches(ctx.handle) - before == 3
        assert d.cpu().numpy().view(np.float32).view(np.uint32).tobytes() == want.view(np.uint32).tobytes()


def test_autotune_picks_a_method_per_bin(ts):
    ctx = ts.Context(0)
    m = ts.segments_autotune(4, ctx)
    assert len(m) == 4 and m[0] in (0, 1, 2, 3, 4) and m[1] in (0, 1, 2, 3, 5) and all(x in (0, 1, 2, 3, 6) for x in m[2:])
    rng = np.random.default_rng(9)
    a, offs = batch("u32", list(rng.integers(0, 20000, size=300)), rng)
    got = a.copy()
    ts.sort_segments(got, offs, ctx)
    assert got.tobytes() == expected(a, offs).tobytes()


def test_warp_methods_only_in_their_bins(ts):
    ctx = ts.Context(0)
    for bad, w in (([0, 4, 0, 0], 4), ([5, 0, 0, 0], 4), ([0, 0, 5, 0], 4), ([0, 5, 0, 0], 8), ([0, 6, 0, 0], 4),
                   ([0, 0, 6, 0], 2)):
        with pytest.raises(ts.TurbosortError):
            ts.segments_methods(w, ctx, bad)


def test_bad_offsets_are_rejected(ts):
    a = np.arange(10, dtype=np.uint32)
    with pytest.raises(ts.TurbosortError):
        ts.sort_segments(a, np.array([0, 5, 3], dtype=np.uint64))
    with pytest.raises(ts.TurbosortError):
        ts.sort_segments(a, np.array([0, 11], dtype=np.uint64))


@pytest.mark.parametrize("t", ["u32", "f32", "i64", "u64", "f64"])
def test_segments_above_the_on_chip_capacity(ts, t):
    """Segments of up to eight times the shared-memory MSD capacity (49.6K
    4-byte or 24.8K 8-byte keys) are cut by key range into parts that fit;
    a part whose narrow key range alone holds too many keys takes the CTA
    LSD. Shapes: random keys, keys crowded into one tiny range with a few
    outliers, two distinct values, and every key equal, at lengths around
    the capacity and its multiples."""
    w = np.dtype(O.NP_DTYPE[t]).itemsize
    cap = 49_600 if w == 4 else 24_800
    rng = np.random.default_rng(77)
    lengths = [cap - 1, cap + 1, 2 * cap + 3, 5 * cap, 8 * cap - 5, 8 * cap + 9, 70_000, 150_000]
    a, offs = batch(t, lengths, rng)
    k = a.view(O.KEY_DTYPE[t])
    lo, hi = int(offs[1]), int(offs[2])            # crowded: 99% of the keys in a 1000-wide range
    k[lo:hi] = np.where(rng.random(hi - lo) < 0.99, rng.integers(0, 1000, size=hi - lo),
                        rng.integers(0, 2**31, size=hi - lo)).astype(k.dtype)
    lo, hi = int(offs[2]), int(offs[3])            # two values
    k[lo:hi] = np.where(rng.random(hi - lo) < 0.5, 3, 12345).astype(k.dtype)
    lo, hi = int(offs[3]), int(offs[4])            # every key equal
    k[lo:hi] = 42
    got = a.copy()
    ts.sort_segments(got, offs)
    assert got.tobytes() == expected(a, offs).tobytes()
