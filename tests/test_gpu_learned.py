"""The learned-partition sort: its output must be bit-exact with the oracle
(the crate's sort) for every key type and distribution, whether the model
is good, absent (the ablation), corrupted, or sends the keys back to the plain
sort; its backward kernel must match the float64 gradient oracle."""
import numpy as np
import pytest

from oracle import learned_oracle as LO
from oracle import oracle as O

pytestmark = pytest.mark.gpu

N = 1 << 21  # above the learned path's 2^20-key floor; the oracle sorts it in well under a second


class _PartitionUnderTest:
    """The package, with the learned sort's cost route off unless a test sets
    it: these tests are about the partition itself, which the route would
    skip for 4-byte keys and for keys the plain sort diverts."""

    def __init__(self, ts):
        self._ts = ts

    def __getattr__(self, name):
        return getattr(self._ts, name)

    def sort_learned(self, a, params=None, ctx=None, **overrides):
        if params is None:
            overrides.setdefault("route_passes", 0)
        return self._ts.sort_learned(a, params, ctx, **overrides)


@pytest.fixture(scope="module")
def ts():
    import turbosort_b200 as ts

    return _PartitionUnderTest(ts)


@pytest.fixture(scope="module")
def W():
    from turbosort_b200 import workloads

    return workloads


def inputs(W, kind, n=N, seed=7):
    rng = np.random.default_rng(seed)
    if kind == "lognormal_f64":
        return W.lognormal_f64(n, seed)
    if kind == "gauss_mix_u64":
        return W.gauss_mix_u64(n, seed)
    if kind == "unit_f32_dups":
        return W.unit_f32_dups(n, seed)
    if kind == "uniform_u32":
        return rng.integers(0, 2**32, size=n, dtype=np.uint64).astype(np.uint32)
    if kind == "uniform_u64":
        return rng.integers(0, 2**64, size=n, dtype=np.uint64)
    if kind == "normal_i32":
        return np.clip(rng.normal(0, 2**24, size=n), -2**31, 2**31 - 1).astype(np.int32)
    if kind == "normal_i64":
        return rng.normal(0, 2.0**50, size=n).astype(np.int64)
    if kind == "specials_f64":
        a = W.lognormal_f64(n, seed) * np.where(rng.random(n) < 0.5, -1.0, 1.0)
        bits = a.view(np.uint64)
        pick = rng.random(n)
        bits[pick < 0.01] = np.uint64(0x7FF8000000000001)
        bits[(pick >= 0.01) & (pick < 0.02)] = np.uint64(0xFFF8000000000000)
        bits[(pick >= 0.02) & (pick < 0.03)] = np.uint64(0x8000000000000000)
        bits[(pick >= 0.03) & (pick < 0.04)] = np.uint64(0)
        bits[(pick >= 0.04) & (pick < 0.045)] = np.uint64(0x7FF0000000000000)
        bits[(pick >= 0.045) & (pick < 0.05)] = np.uint64(0xFFF0000000000000)
        return a
    if kind == "specials_f32":
        a = W.unit_f32_dups(n, seed) * np.where(rng.random(n) < 0.5, -1, 1).astype(np.float32)
        bits = a.view(np.uint32)
        pick = rng.random(n)
        bits[pick < 0.01] = np.uint32(0x7FC00001)
        bits[(pick >= 0.01) & (pick < 0.02)] = np.uint32(0xFFC00000)
        bits[(pick >= 0.02) & (pick < 0.03)] = np.uint32(0x80000000)
        bits[(pick >= 0.03) & (pick < 0.035)] = np.uint32(0x7F800000)
        return a
    raise KeyError(kind)


def same_bits(a, b):
    assert a.dtype == b.dtype and a.shape == b.shape
    w = {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}[a.itemsize]
    bad = np.nonzero(a.view(w) != b.view(w))[0]
    assert bad.size == 0, f"{bad.size} mismatches, first at {bad[:5]}"


KINDS = ["lognormal_f64", "gauss_mix_u64", "unit_f32_dups", "uniform_u32", "uniform_u64", "normal_i32",
         "normal_i64", "specials_f64", "specials_f32"]


@pytest.mark.parametrize("forced", [False, True], ids=["defaults", "partition_forced"])
@pytest.mark.parametrize("kind", KINDS)
def test_learned_exact_host(ts, W, kind, forced):
    """Bit-exact with the oracle; `partition_forced` lifts both fallback
    thresholds so the output always comes from the partition and buckets."""
    a = inputs(W, kind)
    want = O.sort(a)
    got = a.copy()
    extra = {"overflow_factor": 1e9, "max_cdf_error": 1e9} if forced else {}
    st = ts.sort_learned(got, **extra)
    same_bits(got, want)
    assert st["n"] == a.size and st["buckets"] == 1 << 14
    if forced:
        assert st["fell_back"] == 0


@pytest.mark.parametrize("kind", ["lognormal_f64", "gauss_mix_u64", "unit_f32_dups"])
def test_learned_exact_device(ts, W, kind):
    import torch

    a = inputs(W, kind, seed=21)
    want = O.sort(a)
    t = torch.from_numpy(a.copy()).cuda()
    st = ts.sort_learned(t, overflow_factor=1e9, max_cdf_error=1e9)
    torch.cuda.synchronize()
    got = t.cpu().numpy().view(a.dtype)
    same_bits(got, want)
    assert st["fell_back"] == 0, st


@pytest.mark.parametrize("kind", ["lognormal_f64", "gauss_mix_u64", "unit_f32_dups"])
def test_skewed_inputs_stay_balanced(ts, W, kind):
    """At 2^24 keys (about 160 samples a leaf) the fitted model keeps every
    bucket within 4x the mean on the three skewed distributions."""
    a = inputs(W, kind, n=1 << 24)
    st = ts.sort_learned(a)
    assert st["fell_back"] == 0, st
    assert st["imbalance"] < 4.0
    assert st["train_loss_last"] < st["train_loss_first"]
    assert st["max_cdf_error"] < 0.01


def test_ablation_model_vs_equal_width(ts, W):
    """What the trained model gains: on the 8-Gaussian u64 keys equal-width
    buckets put most keys in a few buckets (the input goes back to the plain
    sort), while the model's buckets stay within a small factor of the mean."""
    a = inputs(W, "gauss_mix_u64", n=1 << 24)
    want = O.sort(a)
    with_model = a.copy()
    st_m = ts.sort_learned(with_model)
    without = a.copy()
    st_0 = ts.sort_learned(without, use_model=0)
    same_bits(with_model, want)
    same_bits(without, want)
    assert st_m["fell_back"] == 0 and st_m["imbalance"] < 3.0
    assert st_0["fell_back"] == 1 and st_0["reason"] == 1
    assert st_0["imbalance"] > 10 * st_m["imbalance"]
    # with the fallback threshold lifted the ablation still sorts exactly
    forced = a.copy()
    st_f = ts.sort_learned(forced, use_model=0, overflow_factor=1e9)
    same_bits(forced, want)
    assert st_f["fell_back"] == 0


@pytest.mark.parametrize("kind", ["lognormal_f64", "unit_f32_dups"])
def test_ablation_on_float_keys(ts, W, kind):
    """Float radix keys are already close to a log scale, so equal-width
    buckets do better there than on integers; the model still balances better."""
    a = inputs(W, kind, n=1 << 24)
    st_m = ts.sort_learned(a.copy())
    st_0 = ts.sort_learned(a.copy(), use_model=0, overflow_factor=1e9)
    assert st_m["imbalance"] < st_0["imbalance"]


def test_training_improves_the_fit(ts, W):
    """What the training gains over the same model untrained (train_iters =
    0: heights that interpolate the sample's CDF at the breakpoints): the Adam
    steps lower the mean squared rank error over all of each leaf's samples
    by a third or more on both skewed inputs. That is the whole gain. The
    buckets come out about as even either way (the largest bucket moves by a
    few percent, down on some inputs and up on others: at 2^28 the Gaussian
    mixture's went 2.76x -> 2.38x the mean, the lognormal's 1.77x -> 1.82x),
    and the bucket sorts take the same time, because the untrained leaves
    already start from the sample's quantiles."""
    for kind in ("gauss_mix_u64", "lognormal_f64"):
        a = inputs(W, kind, n=1 << 24)
        st0 = ts.sort_learned(a.copy(), train_iters=0, overflow_factor=1e9)
        st1 = ts.sort_learned(a.copy(), overflow_factor=1e9)
        assert st1["train_iters"] > 0
        assert st0["train_loss_first"] == pytest.approx(st0["train_loss_last"], rel=1e-9)
        assert st1["train_loss_first"] == pytest.approx(st0["train_loss_last"], rel=1e-4)
        assert st1["train_loss_last"] < 0.75 * st1["train_loss_first"]
        assert st1["max_bucket"] <= 1.1 * st0["max_bucket"], (st0["max_bucket"], st1["max_bucket"])


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_corrupted_model_still_exact(ts, W, seed):
    """Leaves overwritten with NaN, +-1e30 and random values: the per-leaf
    bounds keep the bucket map monotone, so the output is still exact."""
    for kind in ("lognormal_f64", "uniform_u32"):
        a = inputs(W, kind, seed=seed)
        want = O.sort(a)
        got = a.copy()
        st = ts.sort_learned(got, corrupt_seed=seed, overflow_factor=1e9, max_cdf_error=1e9)
        same_bits(got, want)
        assert st["fell_back"] == 0


def test_cdf_error_fallback(ts, W):
    a = inputs(W, "lognormal_f64")
    got = a.copy()
    st = ts.sort_learned(got, max_cdf_error=0.0, train_iters=1)
    same_bits(got, O.sort(a))
    assert st["fell_back"] == 1 and st["reason"] in (1, 2)


@pytest.mark.parametrize("n", [0, 1, 2, 1000, (1 << 20) - 1])
def test_small_inputs_take_the_plain_sort(ts, n):
    a = np.random.default_rng(n).lognormal(0, 2, size=n)
    got = a.copy()
    st = ts.sort_learned(got)
    same_bits(got, O.sort(a))
    if n > 1:
        assert st["fell_back"] == 1 and st["reason"] == 3


@pytest.mark.parametrize("blog", [12, 13, 15])
def test_bucket_counts(ts, W, blog):
    a = inputs(W, "gauss_mix_u64", seed=blog)
    got = a.copy()
    st = ts.sort_learned(got, buckets_log2=blog)
    same_bits(got, O.sort(a))
    assert st["buckets"] == 1 << blog


def test_bad_bucket_count_is_rejected(ts):
    a = np.arange(1 << 20, dtype=np.uint64)
    for bad in ({"buckets_log2": 16}, {"buckets_log2": 11}, {"leaves": 1}, {"leaves": 4096},
                {"leaves": 2048, "buckets_log2": 15}):
        with pytest.raises(ts.TurbosortError):
            ts.sort_learned(a, **bad)


def test_lengths_with_constant_and_two_values(ts):
    for a in (np.full(1 << 21, 7, dtype=np.uint64),
              np.where(np.random.default_rng(0).random(1 << 21) < 0.5, 3, 1 << 60).astype(np.uint64)):
        got = a.copy()
        ts.sort_learned(got, overflow_factor=1e9)
        same_bits(got, O.sort(a))


def test_gradients_match_float64_oracle(ts):
    """The backward arithmetic of the training kernel (the same device
    function) against the float64 oracle. Tolerance: float32 products summed
    in float32 over ~100-1000 samples a leaf; each gradient within 1e-4 of the
    largest one plus 1e-3 of its own size."""
    import torch

    rng = np.random.default_rng(5)
    m, leaves, P = 200_000, 1024, LO.P
    cuts = np.sort(rng.choice(np.arange(1, m), size=leaves - 1, replace=False))
    first = np.concatenate([[0], cuts]).astype(np.int32)
    last = np.concatenate([cuts - 1, [m - 1]]).astype(np.int32)
    last[10] = last[11]  # leaf 11 empty, its samples in leaf 10
    first[11] = last[11] = -1
    t = np.zeros(m, np.float32)
    for f, l in zip(first, last):
        if f >= 0:
            t[f:l + 1] = np.sort(rng.random(l - f + 1)).astype(np.float32)
    y = np.sort(rng.random(m)).astype(np.float32)
    bp = np.sort(rng.random((leaves, P - 1)), axis=1).astype(np.float32)
    bp[5, 2:4] = bp[5, 1]  # empty pieces
    y0 = rng.random(leaves).astype(np.float32)
    h = (rng.random(leaves) * 0.01).astype(np.float32)
    v = np.sort(rng.random((leaves, P + 1)), axis=1).astype(np.float32)
    dev = [torch.from_numpy(a).cuda() for a in (t, y, first, last, bp, y0, h, v)]
    g, loss = ts.lm_gradients(*dev)
    rg, rloss = LO.gradients(t, y, first, last, bp, y0, h, v)
    g = g.cpu().numpy().astype(np.float64)
    tol = 1e-4 * np.abs(rg).max() + 1e-3 * np.abs(rg)
    assert np.all(np.abs(g - rg) <= tol), np.abs(g - rg).max()
    assert np.all(g[11] == 0)
    assert abs(loss - rloss) <= 1e-4 * rloss


def test_full_size_equals_plain_sort(ts, W):
    """At the workload's full size (2^28 f64 lognormal keys): the learned sort
    equals the plain device sort bit for bit (the plain sort being pinned to
    the oracle by the other tests), and did not fall back."""
    import torch

    n = 1 << 28
    a = torch.from_numpy(W.lognormal_f64(n, 11)).cuda()
    b = a.clone()
    st = ts.sort_learned(a)
    ts.sort(b)
    torch.cuda.synchronize()
    assert st["fell_back"] == 0, st
    assert torch.equal(a.view(torch.int64), b.view(torch.int64))


@pytest.mark.parametrize("kind, n, routed", [("unit_f32_dups", N, True), ("uniform_u32", N, True),
                                             ("uniform_u64", N, True), ("lognormal_f64", N, None),
                                             ("gauss_mix_u64", 1 << 26, False)])
def test_cost_route(ts, W, kind, n, routed):
    """With the default route, inputs the plain sort handles in at most four
    passes take the plain sort: every 4-byte key, random 8-byte keys (which
    it diverts to four passes), and at 2^21 the lognormal f64 keys, whose top
    digits carry about the 23 bits that diverting needs there (routed when
    the estimate comes to four passes or fewer). At 2^26 the
    Gaussian mixture's top digits split the keys too poorly to divert, all
    eight passes would run, and the partition takes it. The output is the
    oracle's either way."""
    import turbosort_b200 as real

    a = inputs(W, kind, n=n)
    got = a.copy()
    st = real.sort_learned(got)
    same_bits(got, O.sort_parallel(a))
    assert (st["reason"] == 4) == (0 < st["est_plain_passes"] <= 4), st
    if routed is True:
        assert st["fell_back"] == 1 and st["reason"] == 4, st
    elif routed is False:
        assert st["reason"] != 4 and st["est_plain_passes"] >= 5, st


@pytest.mark.parametrize("bits, passes", [(32, 4), (16, 2)])
def test_route_estimate_from_a_short_sample(ts, W, bits, passes):
    """With route_passes = 3, 4-byte keys are sampled and the estimate comes
    from the plain sort of the sample (21K keys here: the single-launch
    sort), which must report each live digit's largest bucket: random u32
    keys need four passes (the partition runs), keys of 16 varying bits two
    (routed to the plain sort)."""
    import turbosort_b200 as real

    rng = np.random.default_rng(bits)
    a = (rng.integers(0, 2**32, size=N, dtype=np.uint64) & np.uint64((1 << bits) - 1)).astype(np.uint32)
    got = a.copy()
    st = real.sort_learned(got, route_passes=3)
    same_bits(got, O.sort(a))
    assert st["est_plain_passes"] == passes, st
    assert (st["reason"] == 4) == (passes <= 3), st


@pytest.mark.parametrize("kind", ["lognormal_f64", "gauss_mix_u64", "unit_f32_dups", "specials_f64"])
def test_verify_compares_with_the_plain_sort(ts, W, kind):
    """verify = 1: the plain LSD sorts a copy on the device and the outputs
    are compared key for key; a good model and a corrupted one both agree."""
    a = inputs(W, kind, seed=33)
    want = O.sort(a)
    for extra in ({}, {"corrupt_seed": 5, "overflow_factor": 1e9, "max_cdf_error": 1e9}):
        got = a.copy()
        st = ts.sort_learned(got, verify=1, **extra)
        same_bits(got, want)
        if st["fell_back"] == 0:
            assert st["verified"] == 1 and st["verify_mismatches"] == 0, st
