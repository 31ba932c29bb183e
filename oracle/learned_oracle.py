"""CPU oracle of the learned partition's model arithmetic — TEST
INFRASTRUCTURE ONLY (imported by tests/ as the checker, never by the product).

The learned partition has no counterpart in the turbosort crate: its output is
pinned to the crate's sort (src/dispatch.rs:31) through the C oracle
(oracle/turbosort_oracle.c), whatever the model does. This file pins the
model's own arithmetic, in float64.

Leaf j owns samples first[j]..last[j]; t_i in [0, 1] is a sample's place in
its leaf, y_i its target CDF value. The leaf is a P-piece linear CDF with
breakpoints 0 <= bp_1 <= ... <= bp_{P-1} <= 1 and heights v_0..v_P:

  piece k     = number of interior breakpoints <= t (0..P-1)
  frac        = (t - left_k) / (right_k - left_k)   (0 for an empty piece)
  prediction  = y0_j + h_j * (v_k + (v_{k+1} - v_k) * frac)
  loss        L = (1/m) sum_i (prediction_i - y_i)^2
  dL/dv_k    += (2/m) R_i h_j (1 - frac),  dL/dv_{k+1} += (2/m) R_i h_j frac

`finite_difference` checks `gradients` against central differences of `loss`,
so the oracle is pinned by the mathematics it restates. `bucket_map` restates
the partition's key -> bucket map (sanitised heights, piece and leaf clamps)
for the monotonicity property.
"""
from __future__ import annotations

import numpy as np

P = 8


def _leaf_of(m, first, last):
    leaf = np.full(m, -1, np.int64)
    for j, (f, l) in enumerate(zip(first, last)):
        if f >= 0:
            leaf[f:l + 1] = j
    assert np.all(leaf >= 0), "every sample must belong to a leaf"
    return leaf


def _pieces(t, bp_rows):
    """piece index and fraction for each t with its leaf's interior breakpoints."""
    t = np.asarray(t, np.float64)
    bp = np.asarray(bp_rows, np.float64)
    k = np.sum(bp <= t[:, None], axis=1)
    left = np.where(k == 0, 0.0, np.take_along_axis(bp, np.maximum(k - 1, 0)[:, None], 1)[:, 0])
    right = np.where(k == P - 1, 1.0, np.take_along_axis(bp, np.minimum(k, P - 2)[:, None], 1)[:, 0])
    width = right - left
    frac = np.where(width > 0, np.clip((t - left) / np.where(width > 0, width, 1), 0, 1), 0.0)
    return k, frac


def predict(t, first, last, bp, y0, h, v):
    m = len(t)
    leaf = _leaf_of(m, first, last)
    bp = np.asarray(bp, np.float64).reshape(-1, P - 1)
    v = np.asarray(v, np.float64).reshape(-1, P + 1)
    k, frac = _pieces(t, bp[leaf])
    vk = v[leaf, k]
    vk1 = v[leaf, k + 1]
    return np.asarray(y0, np.float64)[leaf] + np.asarray(h, np.float64)[leaf] * (vk + (vk1 - vk) * frac), leaf, k, frac


def loss(t, y, first, last, bp, y0, h, v) -> float:
    pred = predict(t, first, last, bp, y0, h, v)[0]
    r = pred - np.asarray(y, np.float64)
    return float(np.mean(r * r))


def gradients(t, y, first, last, bp, y0, h, v):
    """(dL/dv with v's [leaves, P+1] shape, L) in float64."""
    m = len(t)
    pred, leaf, k, frac = predict(t, first, last, bp, y0, h, v)
    r = pred - np.asarray(y, np.float64)
    gr = 2.0 / m * r * np.asarray(h, np.float64)[leaf]
    leaves = len(y0)
    g = np.zeros((leaves, P + 1))
    np.add.at(g, (leaf, k), gr * (1 - frac))
    np.add.at(g, (leaf, k + 1), gr * frac)
    return g, float(np.mean(r * r))


def finite_difference(t, y, first, last, bp, y0, h, v, j: int, q: int, eps: float = 1e-6) -> float:
    """Central difference of `loss` in v[j, q]."""
    w = np.array(v, np.float64).reshape(-1, P + 1)
    w[j, q] += eps
    hi = loss(t, y, first, last, bp, y0, h, w)
    w[j, q] -= 2 * eps
    lo = loss(t, y, first, last, bp, y0, h, w)
    return (hi - lo) / (2 * eps)


def bounds(y0, h, v, bp, empty, buckets):
    """Sanitised heights in bucket units and per-leaf bucket ranges, as the
    partition builds them: NaN dropped, clamps, running maxima."""
    leaves = len(y0)
    c = np.zeros((leaves, P + 1))
    bps = np.zeros((leaves, P - 1))
    a = np.zeros(leaves, np.int64)
    b = np.zeros(leaves, np.int64)
    for j in range(leaves):
        yy, hh = float(y0[j]), float(h[j])
        if np.isnan(yy) or np.isnan(hh):
            yy = hh = 0.0
        yy, hh = min(max(yy, 0.0), 1.0), min(max(hh, 0.0), 1.0)
        prev = 0.0
        for q in range(P - 1):
            x = bp[j][q]
            prev = prev if np.isnan(x) else max(prev, min(x, 1.0))
            bps[j, q] = prev
        pv = pc = 0.0
        for q in range(P + 1):
            x = v[j][q]
            pv = pv if np.isnan(x) else max(pv, min(x, 1.0))
            pc = max(pc, min((yy + hh * pv) * buckets, buckets))
            c[j, q] = pc
        a[j] = min(int(c[j, 0]), buckets - 1)
        b[j] = max(a[j], min(int(c[j, P]), buckets - 1))
        if empty[j]:
            a[j] = b[j] = 0
    hi = np.maximum.accumulate(b)
    lo = np.maximum(a, np.concatenate([[0], hi[:-1]]))
    hi = np.maximum(lo, b)
    return c, bps, lo, np.maximum.accumulate(hi)


def bucket_map(leaf, t, c, bps, lo, hi):
    """Bucket of keys in leaf[] at leaf positions t[] (leaves non-decreasing
    and t non-decreasing within a leaf along the keys)."""
    k, frac = _pieces(t, bps[leaf])
    c0 = c[leaf, k]
    c1 = c[leaf, k + 1]
    b = np.floor(c0 + (c1 - c0) * frac).astype(np.int64)
    b = np.clip(b, np.floor(c0).astype(np.int64), np.floor(c1).astype(np.int64))
    return np.clip(b, lo[leaf], hi[leaf])
