"""Pins the CPU oracle to the turbosort crate's own known answers.

Every vector comes from tests/golden/kat.json, restated from the crate's tests
and docs by tests/golden/make_golden.py (file:line there). The oracle is also
checked against numpy sorts of the radix keys, an independent implementation.
"""
import itertools
import os

import numpy as np
import pytest

from oracle import oracle as O

TYPES = O.TYPES


def bits_as(t, bits):
    kd = O.KEY_DTYPE[t]
    return np.array(bits, dtype=np.uint64).astype(kd).view(O.NP_DTYPE[t])


def test_key_order_i32(kat):
    v = np.array(kat["key_order_i32"], dtype=np.int32)
    k = O.radix_keys(v)
    assert np.all(k[:-1] < k[1:])
    assert np.array_equal(O.from_radix_keys(k, "i32"), v)


def test_key_order_f32(kat):
    v = bits_as("f32", kat["key_order_f32_bits"])
    k = O.radix_keys(v)
    assert np.all(k[:-1] < k[1:])
    rt = O.from_radix_keys(k, "f32").view(np.uint32)
    assert np.array_equal(rt, v.view(np.uint32))


@pytest.mark.parametrize("t", ["f32", "f64"])
def test_total_cmp(kat, t):
    case = kat[f"total_cmp_{t}"]
    v = bits_as(t, case["bits"])
    ib = np.uint32 if t == "f32" else np.uint64
    # round trip on every bit pattern (key.rs:273, :278)
    assert np.array_equal(O.from_radix_keys(O.radix_keys(v), t).view(ib), v.view(ib))
    got = O.sort(v).view(ib)
    assert np.array_equal(got, np.array(case["sorted"], dtype=np.uint64).astype(ib))


@pytest.mark.parametrize("t", ["f32", "f64"])
def test_float_edges(kat, t):
    case = kat[f"float_edge_{t}"]
    ib = np.uint32 if t == "f32" else np.uint64
    got = O.sort(bits_as(t, case["input_bits"])).view(ib)
    assert got.tolist() == case["expected_bits"]


def test_signed_edges(kat):
    for t, case in kat["signed_edge"].items():
        v = np.array(case["input"], dtype=O.NP_DTYPE[t])
        assert O.sort(v).tolist() == case["expected"]


def test_doc_examples(kat):
    for ex in kat["doc_examples"]:
        v = np.array(ex["input"], dtype=O.NP_DTYPE[ex["type"]])
        got = O.sort_with_buffer(v)[0] if ex.get("with_buffer") else O.sort(v)
        assert got.tolist() == ex["expected"]
    case = kat["doc_f32_bits"]
    assert O.sort(bits_as("f32", case["input_bits"])).view(np.uint32).tolist() == case["expected_bits"]


@pytest.mark.parametrize("name", ["by_key_words", "by_key_ids", "by_key_people_age", "by_key_people_name_len"])
def test_by_key_orders(kat, name):
    case = kat[name]
    order = O.sort_by_key_order(np.array(case["keys_u32"], dtype=np.uint32))
    assert order.tolist() == case["order"]


def test_apply_order_example():
    # README.md:61-67: ids [30,10,20] -> order [1,2,0]; names follow.
    order = O.sort_by_key_order(np.array([30, 10, 20], dtype=np.uint32))
    names = np.array([ord("c"), ord("a"), ord("b")], dtype=np.uint8)
    assert O.apply_order(names, order).tolist() == [ord("a"), ord("b"), ord("c")]
    with pytest.raises(ValueError, match="differs from the last sorted slice"):
        O.apply_order(np.array([1, 2], dtype=np.uint8), order)


def test_divert_arithmetic(kat):
    for x, want in kat["log2_eighths"]:
        assert O.log2_eighths(x) == want
    prev = 0
    for x in range(1, 5000):  # divert.rs:279-290
        est = O.log2_eighths(x)
        exact = 8.0 * np.log2(x)
        assert est <= exact + 1e-9 and est > exact - 2.0 and est >= prev
        prev = est
    for c in kat["skippable_digits"]:
        got = O.skippable_digits(c["n_live"], c["len"], [c["max"]] * max(c["n_live"], 1))
        assert got == c["expect"], c


def test_varying_bits(kat):
    vb = kat["varying_bits"]
    assert O.varying_bits(np.array(vb["u64_keys"], dtype=np.uint64)) == vb["u64_expect"]
    assert O.varying_bits(np.array(vb["u32_sevens"], dtype=np.uint32)) == vb["u32_expect"]
    assert O.varying_bits(np.array(vb["u16_keys"], dtype=np.uint16)) is None
    lp = kat["live_passes"]
    assert O.counted_passes_u64(np.array(lp["keys_u64"], dtype=np.uint64)) == lp["live"]


def test_regressions(kat):
    for t in ("f32", "i32"):
        v = np.array(kat["regressions"][t], dtype=O.NP_DTYPE[t])
        want = O.from_radix_keys(np.sort(O.radix_keys(v)), t)
        assert O.sort(v).tobytes() == want.tobytes()


def test_exhaustive_permutations():
    # tests/correctness.rs:12-72: every permutation of u8 0..n (n <= 8) and of
    # i8 -3.. (n <= 6) sorts to the ordered sequence.
    for n in range(0, 9):
        base = list(range(n))
        for p in itertools.permutations(base):
            assert O.sort(np.array(p, dtype=np.uint8)).tolist() == base
    for n in range(0, 7):
        base = list(range(-3, -3 + n))
        for p in itertools.permutations(base):
            assert O.sort(np.array(p, dtype=np.int8)).tolist() == base


def test_xorshift_stream():
    # the first outputs of xorshift64 from the crate's favourite seed
    out, _ = O.xorshift64(0x9E3779B97F4A7C15, 3)
    s = 0x9E3779B97F4A7C15
    m = (1 << 64) - 1
    for v in out:
        s ^= (s << 13) & m
        s ^= s >> 7
        s ^= (s << 17) & m
        assert int(v) == s


@pytest.mark.parametrize("t", TYPES)
def test_oracle_matches_numpy(t):
    """The restated sort, sort_with_buffer, sort_parallel and by_key order agree
    with numpy sorts of the radix keys (an independent implementation) across
    the crate's tier boundaries and key shapes."""
    rng = np.random.default_rng(7)
    kd = O.KEY_DTYPE[t]
    for n in [0, 1, 2, 16, 17, 47, 48, 128, 511, 512, 513, 4096, 70_000, 300_000]:
        for shape in range(5):
            b = rng.integers(0, 2**64, size=n, dtype=np.uint64)
            if shape == 1:
                b %= np.uint64(5)
            elif shape == 2:
                b >>= np.uint64(44)
            elif shape == 3:
                b = np.sort(b)[::-1].copy()
            elif shape == 4:
                b = np.sort(b)
            a = b.astype(kd).view(O.NP_DTYPE[t])
            want = O.from_radix_keys(np.sort(O.radix_keys(a)), t).tobytes()
            assert O.sort(a).tobytes() == want
            assert O.sort_with_buffer(a)[0].tobytes() == want
            assert O.sort_parallel(a, 3).tobytes() == want
            order = O.sort_by_key_order(a)
            assert np.array_equal(order, np.argsort(O.radix_keys(a), kind="stable"))


def test_sort_with_buffer_too_small():
    _, st = O.sort_with_buffer(np.arange(10, dtype=np.uint32), buf_len=9)
    assert st == 1


def test_oracle_under_address_and_undefined_behaviour_sanitizers(tmp_path):
    """The C oracle built with ASan and UBSan (leaks included) and driven
    through every key type, the crate's tier-boundary sizes and shapes, by a
    driver that checks each result itself."""
    import shutil
    import subprocess

    cc = shutil.which("gcc")
    if cc is None:
        pytest.skip("no gcc")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = str(tmp_path / "oracle_sanitize")
    r = subprocess.run([cc, "-std=c11", "-O1", "-g", "-fsanitize=address,undefined", "-fno-sanitize-recover=undefined",
                        os.path.join(root, "oracle", "turbosort_oracle.c"),
                        os.path.join(root, "tests", "cpp", "oracle_sanitize.c"), "-lpthread", "-lm", "-o", exe],
                       capture_output=True, text=True)
    if r.returncode != 0:
        pytest.skip("no sanitizer runtime: " + r.stderr[-200:])
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300,
                       env={**os.environ, "ASAN_OPTIONS": "detect_leaks=1"})
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr[-3000:]


def test_library_divert_rule_matches_the_crate(kat):
    """The diverting rule the device plan applies (k_plan), called on the host
    through the C ABI: the crate's own expected digit counts
    (src/radix/divert.rs:124-148), then the oracle's restatement on random
    histogram maxima."""
    import turbosort_b200 as ts

    for c in kat["skippable_digits"]:
        got = ts.divert_skippable_digits(c["n_live"], c["len"], [c["max"]] * max(c["n_live"], 1))
        assert got == c["expect"], c
    rng = np.random.default_rng(77)
    for _ in range(3000):
        n_live = int(rng.integers(0, 9))
        length = int(rng.integers(1, 1 << 40))
        maxb = [int(rng.integers(1, length + 1)) if rng.random() < 0.3 else max(1, length >> int(rng.integers(0, 12)))
                for _ in range(max(n_live, 1))]
        assert ts.divert_skippable_digits(n_live, length, maxb) == O.skippable_digits(n_live, length, maxb)
