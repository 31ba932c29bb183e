"""Parity of the CUDA sort with the oracle, through the C ABI.

Mirrors the shapes of the crate's tests/correctness.rs (tier boundaries,
structured keys, presorted and reversed input, float and signed edges) and
its by_key tests (src/by_key.rs:368-583). Every comparison is bit-exact.
"""
import zlib

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

TYPES = O.TYPES
SIZES = [2, 3, 15, 16, 17, 47, 48, 100, 128, 511, 512, 513, 1024, 4095, 4096, 4097, 8193, 65553, 300_000]


@pytest.fixture(scope="module")
def ts():
    import turbosort_b200 as ts

    return ts


def gen(t, n, shape, rng):
    kd = O.KEY_DTYPE[t]
    b = rng.integers(0, 2**64, size=n, dtype=np.uint64)
    if shape == "few":
        b %= np.uint64(5)
    elif shape == "low40":
        b >>= np.uint64(24)
    elif shape == "range16":
        b &= np.uint64(0xFFFF)
    elif shape == "and3":
        b &= rng.integers(0, 2**64, size=n, dtype=np.uint64) & rng.integers(0, 2**64, size=n, dtype=np.uint64)
    elif shape == "const":
        b[:] = b[0] if n else 0
    a = b.astype(kd).view(O.NP_DTYPE[t])
    if shape == "asc":
        a = O.sort(a)
    elif shape == "desc":
        a = O.sort(a)[::-1].copy()
    elif shape == "desc_dups":
        a = O.sort((b % np.uint64(97)).astype(kd).view(O.NP_DTYPE[t]))[::-1].copy()
    return a


SHAPES = ["random", "few", "low40", "range16", "and3", "asc", "desc", "desc_dups", "const"]


@pytest.mark.parametrize("t", TYPES)
def test_sort_matches_oracle(ts, t):
    rng = np.random.default_rng(zlib.crc32(t.encode()))
    for n in SIZES:
        for shape in SHAPES:
            a = gen(t, n, shape, rng)
            want = O.sort(a)
            got = a.copy()
            ts.sort(got)
            assert got.tobytes() == want.tobytes(), (t, n, shape)


TORCH_NAME = {"u8": "uint8", "u16": "uint16", "u32": "uint32", "u64": "uint64", "i8": "int8", "i16": "int16",
              "i32": "int32", "i64": "int64", "f32": "float32", "f64": "float64"}
SINT = {1: np.int8, 2: np.int16, 4: np.int32, 8: np.int64}


def to_dev(a, t):
    import torch

    return torch.from_numpy(a.view(SINT[a.itemsize]).copy()).cuda().view(getattr(torch, TORCH_NAME[t]))


def from_dev(d, like):
    import torch

    sint = {1: torch.int8, 2: torch.int16, 4: torch.int32, 8: torch.int64}[like.itemsize]
    return d.view(sint).cpu().numpy().view(like.dtype)


@pytest.mark.parametrize("t", TYPES)
def test_device_sort_matches_oracle(ts, t):
    rng = np.random.default_rng(11)
    for n in [2, 1000, 4097, 100_000, 1 << 20]:
        for shape in ["random", "range16", "desc"]:
            a = gen(t, n, shape, rng)
            want = O.sort(a)
            d = to_dev(a, t)
            ts.sort(d)
            ts.default_context(0).synchronize()
            assert from_dev(d, a).tobytes() == want.tobytes(), (t, n, shape)
            # with a caller's device buffer
            d = to_dev(a, t)
            ts.sort_with_buffer(d, to_dev(np.zeros_like(a), t))
            ts.default_context(0).synchronize()
            assert from_dev(d, a).tobytes() == want.tobytes(), (t, n, shape)


def test_float_specials_at_scale(ts):
    from turbosort_b200 import workloads as W

    for dist in range(3):
        a = W.scale("f32", dist, 3_000_003, seed=99 + dist)
        want = O.sort(a)
        got = a.copy()
        ts.sort(got)
        assert got.view(np.uint32).tobytes() == want.view(np.uint32).tobytes(), dist


def test_golden_vectors_on_gpu(ts, kat):
    for ex in kat["doc_examples"]:
        v = np.array(ex["input"], dtype=O.NP_DTYPE[ex["type"]])
        if ex.get("with_buffer"):
            ts.sort_with_buffer(v, np.zeros_like(v))
        else:
            ts.sort(v)
        assert v.tolist() == ex["expected"]
    for t in ("f32", "f64"):
        case = kat[f"float_edge_{t}"]
        ib = np.uint32 if t == "f32" else np.uint64
        v = np.array(case["input_bits"], dtype=ib).view(O.NP_DTYPE[t])
        ts.sort(v)
        assert v.view(ib).tolist() == case["expected_bits"]
        case = kat[f"total_cmp_{t}"]
        v = np.array(case["bits"], dtype=np.uint64).astype(ib).view(O.NP_DTYPE[t])
        ts.sort(v)
        assert v.view(ib).tolist() == case["sorted"]
    for t, case in kat["signed_edge"].items():
        v = np.array(case["input"], dtype=O.NP_DTYPE[t])
        ts.sort(v)
        assert v.tolist() == case["expected"]
    for t in ("f32", "i32"):
        v = np.array(kat["regressions"][t], dtype=O.NP_DTYPE[t])
        want = O.sort(v)
        ts.sort(v)
        assert v.tobytes() == want.tobytes()


def test_exhaustive_small_permutations(ts):
    import itertools

    for n in range(2, 8):
        for p in itertools.permutations(range(n)):
            v = np.array(p, dtype=np.uint8)
            ts.sort(v)
            assert v.tolist() == list(range(n))
    for n in range(2, 7):
        base = list(range(-3, -3 + n))
        for p in itertools.permutations(base):
            v = np.array(p, dtype=np.int8)
            ts.sort(v)
            assert v.tolist() == base


def test_sort_with_buffer_errors(ts):
    v = np.arange(10, dtype=np.uint32)[::-1].copy()
    with pytest.raises(ValueError, match="buffer too small: need 10, got 9"):
        ts.sort_with_buffer(v, np.zeros(9, dtype=np.uint32))
    ts.sort_with_buffer(v, np.zeros(10, dtype=np.uint32))
    assert v.tolist() == list(range(10))


def test_sort_parallel_matches(ts):
    rng = np.random.default_rng(5)
    for t in ("u32", "u64", "f32", "i16", "u8"):
        a = gen(t, 300_000, "random", rng)
        want = O.sort_parallel(a, 4)
        ts.sort_parallel(a)
        assert a.tobytes() == want.tobytes()


@pytest.mark.parametrize("t", TYPES)
def test_keys_order_matches_oracle(ts, t):
    rng = np.random.default_rng(3)
    for n in [2, 3, 63, 64, 127, 128, 1000, 4096, 4097, 70_000, 300_000]:
        for shape in ["random", "few", "asc", "desc", "desc_dups", "const", "range16"]:
            a = gen(t, n, shape, rng)
            want = O.sort_by_key_order(a)
            got = ts.keys_order(a)
            assert np.array_equal(got, want), (t, n, shape)


def test_by_key_doc_orders(ts, kat):
    for name in ("by_key_words", "by_key_ids", "by_key_people_age", "by_key_people_name_len"):
        keys = np.array(kat[name]["keys_u32"], dtype=np.uint32)
        assert ts.keys_order(keys).tolist() == kat[name]["order"]
    # src/lib.rs:145-147 through the Python mirror of sort_by_key
    people = [("bob", 31), ("alice", 25), ("carol", 31), ("dave", 25)]
    ts.sort_by_key(people, lambda p: np.uint32(p[1]))
    assert people == [("alice", 25), ("dave", 25), ("bob", 31), ("carol", 31)]
    buf = ts.SortByKeyBuffer()
    ts.sort_by_key_with_buffer(people, buf, lambda p: np.uint32(len(p[0])))
    assert people == [("bob", 31), ("dave", 25), ("alice", 25), ("carol", 31)]
    ids = np.array([30, 10, 20], dtype=np.uint32)
    names = ["c", "a", "b"]
    b2 = ts.SortByKeyBuffer()
    ts.sort_by_key_with_buffer(ids, b2, lambda x: x)
    assert b2.order().tolist() == [1, 2, 0]
    b2.apply_order(names)
    assert names == ["a", "b", "c"] and ids.tolist() == [10, 20, 30]
    with pytest.raises(ValueError, match="differs from the last sorted slice"):
        b2.apply_order(["x", "y"])


def test_apply_order_records(ts):
    rng = np.random.default_rng(8)
    n = 200_003
    keys = (rng.integers(0, 1000, size=n)).astype(np.uint64)
    order = ts.keys_order(keys)
    assert np.array_equal(order, O.sort_by_key_order(keys))
    rec = np.zeros(n, dtype=[("id", "<u8"), ("a", "<u4"), ("b", "<u4")])
    rec["id"] = np.arange(n)
    rec["a"] = rng.integers(0, 2**32, size=n, dtype=np.uint64).astype(np.uint32)
    want = O.apply_order(rec.view(np.uint8).reshape(n, 16), order).reshape(-1).view(rec.dtype)
    got = rec.copy()
    ts.apply_order(got, order)
    assert got.tobytes() == want.tobytes()
    # equal keys keep their input order
    k_sorted = keys[got["id"]]
    assert np.all(k_sorted[:-1] <= k_sorted[1:])
    eq = k_sorted[:-1] == k_sorted[1:]
    assert np.all(got["id"][:-1][eq] < got["id"][1:][eq])
    for dt in (np.uint8, np.uint16, np.uint32, np.float64):
        side = rng.integers(0, 200, size=n).astype(dt)
        want = side[order]
        ts.apply_order(side, order)
        assert side.tobytes() == want.tobytes()


def test_device_keys_order(ts):
    import torch

    rng = np.random.default_rng(4)
    keys = rng.integers(0, 50, size=123_457).astype(np.int64)
    want = O.sort_by_key_order(keys)
    d = torch.from_numpy(keys).cuda()
    out = ts.keys_order(d)
    ts.default_context(0).synchronize()
    assert np.array_equal(out.cpu().numpy().view(np.uint32), want)


def test_large_u32_properties(ts):
    """2^26 u32 (bigger than L2): sorted, a permutation (same multiset)."""
    from turbosort_b200 import workloads as W

    a = W.plain_u32(1 << 26, seed=123)
    s = a.copy()
    ts.sort(s)
    assert np.all(s[:-1] <= s[1:])
    assert np.array_equal(np.bincount(a >> 20, minlength=4096), np.bincount(s >> 20, minlength=4096))
    assert int(a.astype(np.uint64).sum()) == int(s.astype(np.uint64).sum())
    assert np.array_equal(np.sort(a), s)


@pytest.mark.parametrize("t", ["u32", "f32", "i64", "u16"])
def test_repeated_sorts_of_one_buffer(ts, t):
    """Repeated device sorts of the same buffer and size replay a captured
    launch sequence (CUDA graph) from the third call on: every call must
    still sort its new contents exactly, including presorted, reversed and
    constant inputs whose plans differ from the captured call's."""
    import torch

    ctx = ts.Context(0)
    rng = np.random.default_rng(23)
    n = (1 << 18) + 7
    d = None
    launches = []
    for shape in ["random", "random", "random", "desc", "asc", "const", "range16", "random"]:
        a = gen(t, n, shape, rng)
        if d is None:
            d = to_dev(a, t)
        else:
            d.copy_(to_dev(a, t))
        torch.cuda.synchronize()  # the copy ran on torch's stream, the sort runs on the context's
        before = ts.lib().ts_ctx_launches(ctx.handle)
        ts.sort(d, ctx)
        ctx.synchronize()
        launches.append(ts.lib().ts_ctx_launches(ctx.handle) - before)
        assert from_dev(d, a).tobytes() == O.sort(a).tobytes(), (t, shape)
    assert len(set(launches)) == 1, launches  # a replay counts the launches it holds
    ctx.close()
    torch.cuda.synchronize()


def test_out_of_memory_is_reported_and_the_context_stays_usable(ts):
    """Forced allocation failure: scratch for 2^40 u64 keys (8 TiB) cannot be
    had; the call reports TS_ERR_OOM with the size it wanted (no fault, no
    sticky error), and the same context sorts as before afterwards."""
    ctx = ts.Context(0)
    a = np.arange(100_000, dtype=np.uint32)[::-1].copy()
    ts.sort(a, ctx)
    with pytest.raises(ts.TurbosortError) as e:
        ctx.reserve(1 << 40, 8)
    assert e.value.status == 5 and "cannot reserve" in str(e.value)
    b = np.random.default_rng(1).integers(0, 2**32, size=300_000, dtype=np.uint64).astype(np.uint32)
    got = b.copy()
    ts.sort(got, ctx)
    assert got.tobytes() == O.sort(b).tobytes()
    ctx.close()
