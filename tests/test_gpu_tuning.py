"""The plain LSD's tile variants and their autotuner.

Every variant the tuner can pick sorts exactly like the oracle, for each key
width it tunes (2, 4 and 8 bytes; unsigned, signed and float transforms), at
lengths in each of its three length bins; the tuner's choice per bin is the
fastest of its candidates (8-bit tile variants, 9-11-bit digits), and the
tuning cache round-trips through its JSON file, takes 8-bit digits from a file
without widths, rejects a width outside 4..11, and is ignored when it was
written on another GPU. Every digit width's parity is in test_gpu_digit_bits.py."""
import json

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LENGTHS = [5_003, 1_000_003, (1 << 22) + 77]  # the small tier edge, then bins 0 and 1


@pytest.fixture(scope="module")
def env():
    import torch

    import turbosort_b200 as ts
    from oracle import oracle as O

    ctx = ts.Context(0)
    return torch, ts, O, ctx


def _keys(t, n, seed):
    rng = np.random.default_rng(seed)
    bits = rng.integers(0, 2**63, size=n, dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, size=n, dtype=np.uint64)
    w = np.dtype(t).itemsize
    return bits.astype({2: np.uint16, 4: np.uint32, 8: np.uint64}[w]).view(t)


@pytest.mark.parametrize("variant", [0, 1, 2])
@pytest.mark.parametrize("t", [np.uint16, np.int16, np.uint32, np.int32, np.float32, np.uint64, np.int64,
                               np.float64])
def test_every_variant_matches_the_oracle(env, variant, t):
    torch, ts, O, ctx = env
    w = np.dtype(t).itemsize
    ctx.lsd_variants(w, [variant] * 3)
    try:
        for i, n in enumerate(LENGTHS):
            a = _keys(t, n, 1000 * variant + 10 * w + i)
            got = a.copy()
            ts.sort(got, ctx)
            assert got.tobytes() == O.sort(a).tobytes(), f"variant {variant} {np.dtype(t)} n={n}"
    finally:
        ctx.lsd_variants(w, [0, 0, 0] if w == 8 else [1, 0, 0])


def test_variant_in_the_largest_bin(env):
    """2^25 + 7 u32 keys (the third bin) through each variant, device-resident."""
    torch, ts, O, ctx = env
    n = (1 << 25) + 7
    a = _keys(np.uint32, n, 99)
    want = O.sort_parallel(a)
    for v in range(3):
        ctx.lsd_variants(4, [v] * 3)
        d = torch.from_numpy(a.view(np.int32)).cuda()
        ts.sort(d.view(torch.uint32), ctx)
        torch.cuda.synchronize()
        assert d.cpu().numpy().view(np.uint32).tobytes() == want.tobytes(), f"variant {v}"
    ctx.lsd_variants(4, [1, 0, 0])


def test_autotune_and_cache(env, tmp_path):
    torch, ts, O, ctx = env
    r = ctx.lsd_autotune(4)
    assert len(r["variants"]) == 3 and all(v in (0, 1, 2) for v in r["variants"])
    assert all(b in (8, 9, 10, 11) for b in r["digit_bits"])
    assert all(ms > 0 for row in r["ms"] for ms in row) and all(len(row) == 6 for row in r["ms"])
    for b, (v, bits) in enumerate(zip(r["variants"], r["digit_bits"])):  # the choice is the fastest measured
        assert r["ms"][b][v if bits == 8 else 3 + bits - 9] == min(r["ms"][b])
    path = str(tmp_path / "tune.json")
    ctx.tune_save(path)
    doc = json.load(open(path))
    assert doc["lsd"]["4"] == r["variants"] and doc["lsd_bits"]["4"] == r["digit_bits"]
    other = ts.Context(0)
    other.lsd_variants(4, [2, 2, 2])
    other.lsd_digit_bits(4, [5, 5, 5])
    assert other.tune_load(path) and other.lsd_variants(4) == r["variants"]
    assert other.lsd_digit_bits(4) == r["digit_bits"]
    # a file written before digit widths were tuned loads with 8-bit digits
    del doc["lsd_bits"]
    json.dump(doc, open(path, "w"))
    other.lsd_digit_bits(4, [5, 5, 5])
    assert other.tune_load(path) and other.lsd_digit_bits(4) == [8, 8, 8]
    doc["lsd_bits"] = {"2": [8, 8, 8], "4": [8, 12, 8], "8": [8, 8, 8]}
    json.dump(doc, open(path, "w"))
    with pytest.raises(ts.TurbosortError):
        other.tune_load(path)
    del doc["lsd_bits"]
    doc["gpu"] = "some other GPU"
    json.dump(doc, open(path, "w"))
    other.lsd_variants(4, [2, 2, 2])
    assert not other.tune_load(path) and other.lsd_variants(4) == [2, 2, 2]
    assert not other.tune_load(str(tmp_path / "missing.json"))
