"""ctypes access to the CPU oracle (libts_oracle.so).

TEST INFRASTRUCTURE ONLY. The oracle is a C restatement of the turbosort
crate's CPU sort (see turbosort_oracle.c for the file:line map). Only tests/,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` import this
module, and only to check or to time the CUDA library against it; the product
package never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libts_oracle.so")

TYPES = ("u8", "u16", "u32", "u64", "i8", "i16", "i32", "i64", "f32", "f64")
NP_DTYPE = {
    "u8": np.uint8, "u16": np.uint16, "u32": np.uint32, "u64": np.uint64,
    "i8": np.int8, "i16": np.int16, "i32": np.int32, "i64": np.int64,
    "f32": np.float32, "f64": np.float64,
}
KEY_DTYPE = {
    "u8": np.uint8, "u16": np.uint16, "u32": np.uint32, "u64": np.uint64,
    "i8": np.uint8, "i16": np.uint16, "i32": np.uint32, "i64": np.uint64,
    "f32": np.uint32, "f64": np.uint64,
}

_lib = None


def build() -> str:
    """Compile the oracle with its Makefile (gcc only)."""
    subprocess.run(["make", "-s", "-C", HERE, "liboracle"], check=True)
    return LIB_PATH


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        vp, sz, i = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int
        for t in TYPES:
            getattr(L, f"tso_sort_{t}").argtypes = [vp, sz]
            getattr(L, f"tso_sort_{t}").restype = None
            getattr(L, f"tso_sort_with_buffer_{t}").argtypes = [vp, sz, vp, sz]
            getattr(L, f"tso_sort_with_buffer_{t}").restype = i
            getattr(L, f"tso_sort_parallel_{t}").argtypes = [vp, sz, i]
            getattr(L, f"tso_sort_parallel_{t}").restype = None
            getattr(L, f"tso_sort_by_key_{t}").argtypes = [vp, sz, vp]
            getattr(L, f"tso_sort_by_key_{t}").restype = i
            getattr(L, f"tso_radix_keys_{t}").argtypes = [vp, vp, sz]
            getattr(L, f"tso_from_radix_keys_{t}").argtypes = [vp, vp, sz]
            getattr(L, f"tso_varying_bits_{t}").argtypes = [vp, sz, ctypes.POINTER(ctypes.c_uint64)]
            getattr(L, f"tso_varying_bits_{t}").restype = i
        L.tso_log2_eighths.argtypes = [sz]
        L.tso_log2_eighths.restype = ctypes.c_uint32
        L.tso_skippable_digits.argtypes = [sz, sz, vp]
        L.tso_skippable_digits.restype = sz
        L.tso_apply_order.argtypes = [vp, sz, sz, vp, sz]
        L.tso_apply_order.restype = i
        L.tso_counted_passes_u64.argtypes = [vp, sz, vp]
        L.tso_counted_passes_u64.restype = i
        L.tso_xorshift64_fill.argtypes = [ctypes.POINTER(ctypes.c_uint64), vp, sz]
        _lib = L
    return _lib


def type_of(a: np.ndarray) -> str:
    for t, d in NP_DTYPE.items():
        if a.dtype == np.dtype(d):
            return t
    raise TypeError(f"not a sortable dtype: {a.dtype}")


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def sort(a: np.ndarray) -> np.ndarray:
    """turbosort::sort (lib.rs:99) on a copy; returns the sorted copy."""
    out = np.ascontiguousarray(a).copy()
    getattr(lib(), f"tso_sort_{type_of(out)}")(_ptr(out), out.size)
    return out


def sort_with_buffer(a: np.ndarray, buf_len: int | None = None) -> tuple[np.ndarray, int]:
    """turbosort::sort_with_buffer (lib.rs:122); returns (sorted copy, status)."""
    out = np.ascontiguousarray(a).copy()
    n = out.size if buf_len is None else buf_len
    buf = np.empty(max(n, 1), dtype=out.dtype)
    st = getattr(lib(), f"tso_sort_with_buffer_{type_of(out)}")(_ptr(out), out.size, _ptr(buf), n)
    return out, st


def sort_parallel(a: np.ndarray, threads: int | None = None) -> np.ndarray:
    """turbosort::sort_parallel (lib.rs:224) on a copy."""
    out = np.ascontiguousarray(a).copy()
    sort_parallel_inplace(out, threads)
    return out


def sort_parallel_inplace(a: np.ndarray, threads: int | None = None) -> None:
    th = threads or os.cpu_count() or 1
    getattr(lib(), f"tso_sort_parallel_{type_of(a)}")(_ptr(a), a.size, th)


def sort_inplace(a: np.ndarray) -> None:
    getattr(lib(), f"tso_sort_{type_of(a)}")(_ptr(a), a.size)


def sort_by_key_order(keys: np.ndarray) -> np.ndarray | None:
    """order() after sort_by_key_with_buffer (by_key.rs:175); None if left empty."""
    k = np.ascontiguousarray(keys)
    order = np.empty(max(k.size, 1), dtype=np.uint32)
    st = getattr(lib(), f"tso_sort_by_key_{type_of(k)}")(_ptr(k), k.size, _ptr(order))
    return None if st else order[: k.size]


def apply_order(data: np.ndarray, order: np.ndarray) -> np.ndarray:
    """SortByKeyBuffer::apply_order (by_key.rs:136) on a copy of `data`."""
    out = np.ascontiguousarray(data).copy()
    o = np.ascontiguousarray(order, dtype=np.uint32)
    st = lib().tso_apply_order(_ptr(out), out.shape[0] if out.ndim else 0,
                               out.itemsize * (out[0].size if out.ndim > 1 else 1),
                               _ptr(o), o.size)
    if st:
        raise ValueError("apply_order: the slice's length differs from the last sorted slice's")
    return out


def radix_keys(a: np.ndarray) -> np.ndarray:
    """to_radix_key (key.rs:53-62) element-wise."""
    a = np.ascontiguousarray(a)
    t = type_of(a)
    out = np.empty(a.size, dtype=KEY_DTYPE[t])
    getattr(lib(), f"tso_radix_keys_{t}")(_ptr(a), _ptr(out), a.size)
    return out


def from_radix_keys(k: np.ndarray, t: str) -> np.ndarray:
    k = np.ascontiguousarray(k, dtype=KEY_DTYPE[t])
    out = np.empty(k.size, dtype=NP_DTYPE[t])
    getattr(lib(), f"tso_from_radix_keys_{t}")(_ptr(k), _ptr(out), k.size)
    return out


def varying_bits(a: np.ndarray):
    """histogram::varying_bits (histogram.rs:55); None when every byte varies."""
    a = np.ascontiguousarray(a)
    v = ctypes.c_uint64(0)
    some = getattr(lib(), f"tso_varying_bits_{type_of(a)}")(_ptr(a), a.size, ctypes.byref(v))
    return int(v.value) if some else None


def counted_passes_u64(keys: np.ndarray) -> list[int]:
    k = np.ascontiguousarray(keys, dtype=np.uint64)
    out = np.zeros(8, dtype=np.int32)
    m = lib().tso_counted_passes_u64(_ptr(k), k.size, _ptr(out))
    return [int(x) for x in out[:m]]


def log2_eighths(x: int) -> int:
    return int(lib().tso_log2_eighths(x))


def skippable_digits(n_live: int, length: int, max_buckets) -> int:
    mb = np.ascontiguousarray(np.asarray(list(max_buckets) or [0], dtype=np.uint64))
    return int(lib().tso_skippable_digits(n_live, length, _ptr(mb)))


def xorshift64(seed: int, n: int) -> tuple[np.ndarray, int]:
    """n outputs of the crate's test xorshift64 (13/7/17) and the next state."""
    st = ctypes.c_uint64(seed)
    out = np.empty(max(n, 1), dtype=np.uint64)
    lib().tso_xorshift64_fill(ctypes.byref(st), _ptr(out), n)
    return out[:n], int(st.value)
