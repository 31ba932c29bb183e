"""The learned model's float64 oracle, pinned by the mathematics it restates:
its analytic gradients agree with central differences of its loss, and the
partition's bucket map is non-decreasing for any parameter values (the
property that keeps the learned sort exact)."""
import numpy as np
import pytest

from oracle import learned_oracle as LO

P = LO.P


def problem(seed, m=3000, leaves=12):
    rng = np.random.default_rng(seed)
    cuts = np.sort(rng.choice(np.arange(1, m), size=leaves - 1, replace=False))
    first = np.concatenate([[0], cuts])
    last = np.concatenate([cuts - 1, [m - 1]])
    last[2] = last[3]  # leaf 3 empty: its samples go to leaf 2
    first[3] = last[3] = -1
    t = np.zeros(m)
    for f, l in zip(first, last):
        if f >= 0:
            t[f:l + 1] = np.sort(rng.random(l - f + 1))
    y = np.sort(rng.random(m))
    bp = np.sort(rng.random((leaves, P - 1)), axis=1)
    y0 = rng.random(leaves)
    h = rng.random(leaves) * 0.1
    v = np.sort(rng.random((leaves, P + 1)), axis=1)
    return t, y, first, last, bp, y0, h, v


@pytest.mark.parametrize("seed", range(4))
def test_gradients_equal_finite_differences(seed):
    args = problem(seed)
    g, L = LO.gradients(*args)
    assert L == pytest.approx(LO.loss(*args))
    rng = np.random.default_rng(seed + 100)
    for _ in range(12):
        j, q = int(rng.integers(0, 12)), int(rng.integers(0, P + 1))
        assert g[j, q] == pytest.approx(LO.finite_difference(*args, j, q), rel=1e-5, abs=1e-11)


def test_gradient_of_an_empty_leaf_is_zero():
    t, y, first, last, bp, y0, h, v = problem(9)
    g, _ = LO.gradients(t, y, first, last, bp, y0, h, v)
    assert np.all(g[3] == 0)


@pytest.mark.parametrize("seed", range(8))
def test_bucket_map_is_monotone_for_any_parameters(seed):
    rng = np.random.default_rng(seed)
    leaves, buckets = 40, 1024
    hostile = np.array([np.nan, -1e30, 1e30, 0.0, 0.5, -3.0, 2.0])
    y0 = rng.choice(hostile, leaves) * rng.random(leaves)
    h = rng.choice(hostile, leaves) * rng.random(leaves)
    v = rng.choice(hostile, (leaves, P + 1)) * rng.random((leaves, P + 1))
    bp = rng.choice(hostile, (leaves, P - 1)) * rng.random((leaves, P - 1))
    empty = rng.random(leaves) < 0.1
    c, bps, lo, hi = LO.bounds(y0, h, v, bp, empty, buckets)
    # keys in order: leaves non-decreasing, t non-decreasing inside a leaf
    leaf = np.sort(rng.integers(0, leaves, 20000))
    leaf = leaf[~empty[leaf]]
    t = np.zeros(leaf.size)
    for j in np.unique(leaf):
        sel = leaf == j
        t[sel] = np.sort(rng.random(sel.sum()))
    b = LO.bucket_map(leaf, t, c, bps, lo, hi)
    assert np.all(np.diff(b) >= 0)
    assert b.min() >= 0 and b.max() < buckets
