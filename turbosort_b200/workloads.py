"""Seeded synthetic inputs with the shapes of the benchmark configurations.

    plain_u32(n)              2^20 (or any n) u32 of 32 random bits each
    scale(kind, dist, n)      u32/i32/f32/u64 at scale; dist 0 full entropy,
                              1 AND of three words, 2 confined to 16 low bits;
                              f32 mixes in 1% NaN, 1% +-0.0, 0.5% +-inf
    zipf_u64(n)               by-key keys: Zipf(s=1.1) over 2^20 distinct values
    segment_lengths(count)    log-uniform segment lengths on [1, 65536]
    lognormal_f64 / gauss_mix_u64 / unit_f32_dups   the learned-partition inputs

The first two use the crate's xorshift64 through libts_workloads.so; the rest
use numpy's PCG64 with the given seed.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(PKG, "libts_workloads.so")
SEED = 0x9E3779B97F4A7C15
_w = None


def _lib():
    global _w
    if _w is None:
        if not os.path.exists(_LIB):
            from . import build as _b

            _b.build()
        L = ctypes.CDLL(_LIB)
        vp, sz, u64 = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint64
        L.tsw_gen_u32.argtypes = [u64, ctypes.c_int, vp, sz]
        L.tsw_gen_u64.argtypes = [u64, ctypes.c_int, vp, sz]
        L.tsw_gen_f32_bits.argtypes = [u64, ctypes.c_int, vp, sz]
        L.tsw_xorshift64.argtypes = [ctypes.POINTER(u64), vp, sz]
        _w = L
    return _w


def xorshift64(seed: int, n: int) -> np.ndarray:
    st = ctypes.c_uint64(seed)
    out = np.empty(max(n, 1), dtype=np.uint64)
    _lib().tsw_xorshift64(ctypes.byref(st), out.ctypes.data, n)
    return out[:n]


def plain_u32(n: int = 1 << 20, seed: int = SEED, out: np.ndarray | None = None) -> np.ndarray:
    out = np.empty(n, dtype=np.uint32) if out is None else out
    _lib().tsw_gen_u32(seed, 0, out.ctypes.data, n)
    return out


DISTS = ("full", "low_entropy", "range16")
KINDS = ("u32", "i32", "f32", "u64")


def scale(kind: str, dist: int | str, n: int, seed: int = SEED, out: np.ndarray | None = None) -> np.ndarray:
    d = DISTS.index(dist) if isinstance(dist, str) else int(dist)
    if kind == "u64":
        out = np.empty(n, dtype=np.uint64) if out is None else out
        _lib().tsw_gen_u64(seed, d, out.ctypes.data, n)
        return out
    if kind == "f32":
        buf = np.empty(n, dtype=np.uint32) if out is None else out.view(np.uint32)
        _lib().tsw_gen_f32_bits(seed, d, buf.ctypes.data, n)
        return buf.view(np.float32)
    buf = np.empty(n, dtype=np.uint32) if out is None else out.view(np.uint32)
    _lib().tsw_gen_u32(seed, d, buf.ctypes.data, n)
    return buf.view(np.int32) if kind == "i32" else buf


def zipf_u64(n: int, distinct: int = 1 << 20, s: float = 1.1, seed: int = 3) -> np.ndarray:
    """Keys drawn Zipf(s) over `distinct` random u64 values (rank -> value
    table; rank by inverse CDF)."""
    rng = np.random.default_rng(seed)
    values = rng.integers(0, 2**64, size=distinct, dtype=np.uint64)
    w = 1.0 / np.arange(1, distinct + 1, dtype=np.float64) ** s
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    u = rng.random(n)
    ranks = np.minimum(np.searchsorted(cdf, u, side="right"), distinct - 1)
    return values[ranks]


def segment_lengths(count: int = 100_000, max_len: int = 65536, seed: int = 5) -> np.ndarray:
    rng = np.random.default_rng(seed)
    u = rng.random(count)
    return np.maximum(1, np.floor(np.exp(u * np.log(max_len)))).astype(np.int64)


def lognormal_f64(n: int, seed: int = 11) -> np.ndarray:
    return np.random.default_rng(seed).lognormal(0.0, 2.0, size=n)


def gauss_mix_u64(n: int, seed: int = 13) -> np.ndarray:
    rng = np.random.default_rng(seed)
    means = rng.random(8) * 2.0**60
    comp = rng.integers(0, 8, size=n)
    x = rng.normal(means[comp], 2.0**40)
    x = np.clip(x, 0.0, 2.0**64 - 4096.0)
    return x.astype(np.uint64)


def unit_f32_dups(n: int, seed: int = 17) -> np.ndarray:
    rng = np.random.default_rng(seed)
    x = rng.random(n, dtype=np.float32)
    m = rng.random(n) < 0.10
    idx = np.nonzero(m)[0]
    src = (rng.random(idx.size) * np.maximum(idx, 1)).astype(np.int64)
    x[idx] = x[src]
    return x
