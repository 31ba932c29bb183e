"""turbosort_b200 — the turbosort crate's sort API on a B200, over its C ABI.

Mirrors the crate's public functions (src/lib.rs) for numpy arrays (host
slices: copied to the GPU, sorted there, copied back) and CUDA torch tensors
(device slices: sorted in place on the context's stream):

    sort(a)                      src/lib.rs:99
    sort_with_buffer(a, buf)     src/lib.rs:122   ValueError "buffer too small: need N, got M"
    sort_parallel(a)             src/lib.rs:224
    sort_by_key(items, key)      src/lib.rs:152   stable; key called once per element
    sort_by_key_with_buffer(items, buffer, key)   src/lib.rs:196
    SortByKeyBuffer.order() / .apply_order(other) / .capacity()   src/by_key.rs:51-145

and adds the batched segmented sort (sort_segments) and the learned-partition
sort (sort_learned), whose outputs equal the crate's sort of each slice.

Every call goes through libturbosort_b200.so (include/turbosort.h); there is
no CPU fallback: without the library or a CUDA device the calls raise.
"""
from __future__ import annotations

import ctypes
import os
import threading

import numpy as np

__all__ = [
    "Context", "SortByKeyBuffer", "TurbosortError", "apply_order", "default_context", "lib", "sort",
    "sort_by_key", "sort_by_key_with_buffer", "sort_parallel", "sort_segments", "sort_with_buffer", "segments_autotune",
    "segments_methods", "TYPES", "LearnedParams", "LearnedStats", "learned_params", "lm_gradients", "sort_learned",
    "SortInfo", "divert_skippable_digits", "lsd_variant_ipt",
]

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libturbosort_b200.so")

TYPES = ("u8", "u16", "u32", "u64", "i8", "i16", "i32", "i64", "f32", "f64")
_NP = {
    "u8": np.uint8, "u16": np.uint16, "u32": np.uint32, "u64": np.uint64,
    "i8": np.int8, "i16": np.int16, "i32": np.int32, "i64": np.int64,
    "f32": np.float32, "f64": np.float64,
}
_TORCH_NAME = {
    "uint8": "u8", "uint16": "u16", "uint32": "u32", "uint64": "u64", "int8": "i8", "int16": "i16",
    "int32": "i32", "int64": "i64", "float32": "f32", "float64": "f64",
}

TS_OK = 0
STATUS = {
    1: "TS_ERR_BUFFER_TOO_SMALL", 2: "TS_ERR_LENGTH_MISMATCH", 3: "TS_ERR_CUDA", 4: "TS_ERR_TIMEOUT",
    5: "TS_ERR_OOM", 6: "TS_ERR_INVALID", 7: "TS_ERR_NO_DEVICE", 8: "TS_ERR_TOO_LARGE", 9: "TS_ERR_INTERNAL",
}


LEARNED_TYPES = ("u32", "u64", "i32", "i64", "f32", "f64")


class LearnedParams(ctypes.Structure):
    """ts_learned_params: bucket count, sample rate, model size, training and
    fallback thresholds of the learned-partition sort."""
    _fields_ = [("buckets_log2", ctypes.c_uint32), ("sample_every", ctypes.c_uint32), ("leaves", ctypes.c_uint32),
                ("train_iters", ctypes.c_uint32), ("lr", ctypes.c_float), ("overflow_factor", ctypes.c_float),
                ("max_cdf_error", ctypes.c_float), ("use_model", ctypes.c_int32), ("corrupt_seed", ctypes.c_uint64),
                ("route_passes", ctypes.c_uint32), ("verify", ctypes.c_int32)]


class LearnedStats(ctypes.Structure):
    """ts_learned_stats: what the learned-partition sort did."""
    _fields_ = [("n", ctypes.c_uint64), ("sample_size", ctypes.c_uint64), ("buckets", ctypes.c_uint64),
                ("max_bucket", ctypes.c_uint64), ("mean_bucket", ctypes.c_double), ("imbalance", ctypes.c_double),
                ("train_loss_first", ctypes.c_double), ("train_loss_last", ctypes.c_double),
                ("max_cdf_error", ctypes.c_float), ("train_iters", ctypes.c_uint32), ("fell_back", ctypes.c_int32),
                ("reason", ctypes.c_int32), ("ms_sample", ctypes.c_float), ("ms_train", ctypes.c_float),
                ("ms_partition", ctypes.c_float), ("ms_buckets", ctypes.c_float),
                ("est_plain_passes", ctypes.c_int32), ("verified", ctypes.c_int32),
                ("verify_mismatches", ctypes.c_uint64), ("ms_verify", ctypes.c_float), ("pad", ctypes.c_float)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class SortInfo(ctypes.Structure):
    """ts_sort_info: what the context's last plain sort did."""
    _fields_ = [("tier", ctypes.c_int32), ("mode", ctypes.c_int32), ("passes", ctypes.c_int32),
                ("divert_shift", ctypes.c_int32), ("pass_digit", ctypes.c_int32 * 16), ("digit_bits", ctypes.c_int32)]

    def as_dict(self) -> dict:
        return {"tier": self.tier, "mode": self.mode, "passes": self.passes, "divert_shift": self.divert_shift,
                "pass_digit": list(self.pass_digit[:self.passes]), "digit_bits": self.digit_bits}


def lsd_variant_ipt(key_bytes: int, variant: int) -> int:
    """Keys a thread of a plain-LSD tile variant."""
    return int(lib().ts_lsd_variant_ipt(key_bytes, variant))


def divert_skippable_digits(n_live: int, length: int, max_buckets) -> int:
    """The library's diverting rule (src/radix/divert.rs:38-54), host-side."""
    arr = (ctypes.c_uint64 * max(1, len(max_buckets)))(*[int(x) for x in max_buckets])
    return int(lib().ts_divert_skippable_digits(n_live, length, arr))


class TurbosortError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


_lib = None
_lib_lock = threading.Lock()


def lib() -> ctypes.CDLL:
    """The loaded C ABI library. Raises if it has not been built."""
    global _lib
    with _lib_lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise ImportError(
                    f"{LIB_PATH} is missing: build it with `python -m turbosort_b200.build` (nvcc, sm_100a)")
            L = ctypes.CDLL(LIB_PATH)
            vp, sz, i, st = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_int
            L.ts_ctx_create.argtypes = [i, ctypes.POINTER(vp)]
            L.ts_ctx_create.restype = st
            L.ts_ctx_destroy.argtypes = [vp]
            L.ts_ctx_destroy.restype = None
            L.ts_ctx_set_stream.argtypes = [vp, vp]
            L.ts_ctx_set_stream.restype = st
            L.ts_ctx_stream.argtypes = [vp]
            L.ts_ctx_stream.restype = vp
            L.ts_ctx_synchronize.argtypes = [vp]
            L.ts_ctx_synchronize.restype = st
            L.ts_ctx_reserve.argtypes = [vp, sz, sz, i]
            L.ts_ctx_reserve.restype = st
            L.ts_ctx_capacity.argtypes = [vp, sz, i]
            L.ts_ctx_capacity.restype = sz
            L.ts_ctx_last_error.argtypes = [vp]
            L.ts_ctx_last_error.restype = ctypes.c_char_p
            L.ts_status_str.argtypes = [st]
            L.ts_status_str.restype = ctypes.c_char_p
            L.ts_ctx_enable_timing.argtypes = [vp, i]
            L.ts_ctx_enable_timing.restype = st
            L.ts_ctx_timings.argtypes = [vp, vp, vp, vp, i]
            L.ts_ctx_timings.restype = i
            L.ts_ctx_reset_timings.argtypes = [vp]
            L.ts_ctx_reset_timings.restype = None
            for t in TYPES:
                for name, args in (
                    ("ts_sort_", [vp, vp, sz]),
                    ("ts_sort_with_buffer_", [vp, vp, sz, vp, sz]),
                    ("ts_sort_parallel_", [vp, vp, sz]),
                    ("ts_sort_keys_order_", [vp, vp, sz, vp]),
                    ("ts_sort_dev_", [vp, vp, sz]),
                    ("ts_sort_dev_with_buffer_", [vp, vp, sz, vp, sz]),
                    ("ts_sort_keys_order_dev_", [vp, vp, sz, vp]),
                ):
                    f = getattr(L, name + t)
                    f.argtypes = args
                    f.restype = st
            for t in TYPES:
                getattr(L, f"ts_sort_segments_{t}").argtypes = [vp, vp, sz, vp, sz]
                getattr(L, f"ts_sort_segments_{t}").restype = st
                getattr(L, f"ts_sort_segments_dev_{t}").argtypes = [vp, vp, sz, vp, sz]
                getattr(L, f"ts_sort_segments_dev_{t}").restype = st
            L.ts_segments_autotune.argtypes = [vp, sz]
            L.ts_segments_autotune.restype = st
            L.ts_segments_methods.argtypes = [vp, sz, vp, i]
            L.ts_segments_methods.restype = st
            L.ts_ctx_transfer_pipeline.argtypes = [vp, i, sz]
            L.ts_ctx_transfer_pipeline.restype = st
            L.ts_ctx_use_graphs.argtypes = [vp, i]
            L.ts_ctx_use_graphs.restype = st
            L.ts_ctx_launches.argtypes = [vp]
            L.ts_ctx_launches.restype = ctypes.c_ulonglong
            L.ts_ctx_last_sort_info.argtypes = [vp, ctypes.POINTER(SortInfo)]
            L.ts_ctx_last_sort_info.restype = st
            L.ts_lsd_autotune.argtypes = [vp, sz, ctypes.POINTER(ctypes.c_float)]
            L.ts_lsd_autotune.restype = st
            L.ts_lsd_variants.argtypes = [vp, sz, ctypes.POINTER(ctypes.c_int), i]
            L.ts_lsd_variants.restype = st
            L.ts_lsd_variant_ipt.argtypes = [sz, i]
            L.ts_lsd_variant_ipt.restype = i
            L.ts_lsd_digit_bits.argtypes = [vp, sz, ctypes.POINTER(ctypes.c_int), i]
            L.ts_lsd_digit_bits.restype = st
            L.ts_ctx_tune_save.argtypes = [vp, ctypes.c_char_p]
            L.ts_ctx_tune_save.restype = st
            L.ts_ctx_tune_load.argtypes = [vp, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int)]
            L.ts_ctx_tune_load.restype = st
            L.ts_ctx_set_divert.argtypes = [vp, i]
            L.ts_ctx_set_divert.restype = st
            L.ts_ctx_set_single_launch.argtypes = [vp, i]
            L.ts_ctx_set_single_launch.restype = st
            L.ts_ctx_test_stall_lookback.argtypes = [vp, ctypes.c_uint32]
            L.ts_ctx_test_stall_lookback.restype = st
            L.ts_divert_skippable_digits.argtypes = [i, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64)]
            L.ts_divert_skippable_digits.restype = i
            L.ts_apply_order.argtypes = [vp, vp, sz, sz, vp, sz]
            L.ts_apply_order.restype = st
            L.ts_apply_order_dev.argtypes = [vp, vp, sz, sz, vp, sz]
            L.ts_apply_order_dev.restype = st
            for t in LEARNED_TYPES:
                for name in ("ts_sort_learned_", "ts_sort_learned_dev_"):
                    f = getattr(L, name + t)
                    f.argtypes = [vp, vp, sz, ctypes.POINTER(LearnedParams), ctypes.POINTER(LearnedStats)]
                    f.restype = st
            L.ts_learned_defaults.argtypes = [ctypes.POINTER(LearnedParams)]
            L.ts_learned_defaults.restype = None
            L.ts_lm_gradients.argtypes = [vp, vp, vp, sz, i, vp, vp, vp, vp, vp, vp, vp,
                                          ctypes.POINTER(ctypes.c_double)]
            L.ts_lm_gradients.restype = st
            _lib = L
        return _lib


class Context:
    """A CUDA stream plus device scratch that grows to the largest sort."""

    def __init__(self, device: int = 0):
        self._h = ctypes.c_void_p()
        self._check(lib().ts_ctx_create(device, ctypes.byref(self._h)))
        self.device = device

    def _check(self, status: int) -> None:
        if status != TS_OK:
            msg = lib().ts_ctx_last_error(self._h).decode() if getattr(self, "_h", None) else ""
            if status == 1:
                raise ValueError(msg)
            if status == 2:
                raise ValueError(msg)
            raise TurbosortError(status, msg or lib().ts_status_str(status).decode())

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    def close(self) -> None:
        if self._h:
            lib().ts_ctx_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_handle: int | None) -> None:
        self._check(lib().ts_ctx_set_stream(self._h, stream_handle or None))

    def synchronize(self) -> None:
        self._check(lib().ts_ctx_synchronize(self._h))

    def reserve(self, n: int, key_bytes: int, with_order: bool = False) -> None:
        self._check(lib().ts_ctx_reserve(self._h, n, key_bytes, int(with_order)))

    def capacity(self, key_bytes: int, with_order: bool = False) -> int:
        return int(lib().ts_ctx_capacity(self._h, key_bytes, int(with_order)))

    def transfer_pipeline(self, chunks: int = 8, min_bytes: int = 64 << 20) -> None:
        """Host-slice sorts of at least min_bytes cross PCIe as `chunks` pieces,
        sorted and merged on the device while the copies run (1 turns it off)."""
        self._check(lib().ts_ctx_transfer_pipeline(self._h, chunks, min_bytes))

    def lsd_autotune(self, key_bytes: int) -> dict:
        """Time every 8-bit onesweep tile variant and the 9-, 10- and 11-bit
        digit widths per length bin for keys of this width and keep the
        fastest; returns the choices and the times (per bin: the three 8-bit
        variants, then 9, 10 and 11 bits)."""
        ms = (ctypes.c_float * 18)()
        self._check(lib().ts_lsd_autotune(self._h, key_bytes, ms))
        v = self.lsd_variants(key_bytes)
        return {"variants": v, "keys_per_thread": [lsd_variant_ipt(key_bytes, x) for x in v],
                "digit_bits": self.lsd_digit_bits(key_bytes),
                "ms": [[round(ms[b * 6 + x], 4) for x in range(6)] for b in range(3)],
                "bins": ["n < 2^22", "n < 2^25", "larger"]}

    def lsd_digit_bits(self, key_bytes: int, bits=None) -> list[int]:
        """The plain LSD's digit width (4..11) per length bin for this key
        width (set when given; widths other than 8 apply to keys-only sorts
        below 2^31 keys)."""
        arr = (ctypes.c_int * 3)(*(bits or [8, 8, 8]))
        self._check(lib().ts_lsd_digit_bits(self._h, key_bytes, arr, int(bits is not None)))
        return list(arr)

    def lsd_variants(self, key_bytes: int, variants=None) -> list[int]:
        """The tile variant per length bin for this key width (set when given)."""
        arr = (ctypes.c_int * 3)(*(variants or [0, 0, 0]))
        self._check(lib().ts_lsd_variants(self._h, key_bytes, arr, int(variants is not None)))
        return list(arr)

    def tune_save(self, path: str) -> None:
        self._check(lib().ts_ctx_tune_save(self._h, os.fsencode(path)))

    def tune_load(self, path: str) -> bool:
        loaded = ctypes.c_int(0)
        self._check(lib().ts_ctx_tune_load(self._h, os.fsencode(path), ctypes.byref(loaded)))
        return bool(loaded.value)

    def set_single_launch(self, on: bool) -> None:
        """Sorts of 2- and 4-byte keys whose tiles fit one wave run in one
        cooperative launch (on by default); off, they take the multi-launch LSD."""
        self._check(lib().ts_ctx_set_single_launch(self._h, int(on)))

    def set_divert(self, on: bool) -> None:
        """Diverting of 8-byte keys (on by default); off, every live digit gets a pass."""
        self._check(lib().ts_ctx_set_divert(self._h, int(on)))

    def last_sort_info(self) -> dict:
        """Tier, mode, scatter passes and divert shift of the last plain sort."""
        info = SortInfo()
        self._check(lib().ts_ctx_last_sort_info(self._h, ctypes.byref(info)))
        return info.as_dict()

    def enable_timing(self, on: bool = True) -> None:
        self._check(lib().ts_ctx_enable_timing(self._h, int(on)))

    def reset_timings(self) -> None:
        lib().ts_ctx_reset_timings(self._h)

    def timings(self) -> dict[str, tuple[float, int]]:
        """{kernel group: (total ms, launches)} since the last reset."""
        m = 64
        names = (ctypes.c_char * 32 * m)()
        ms = (ctypes.c_double * m)()
        cnt = (ctypes.c_long * m)()
        k = lib().ts_ctx_timings(self._h, names, ms, cnt, m)
        return {bytes(names[i]).split(b"\0")[0].decode(): (ms[i], cnt[i]) for i in range(min(k, m))}


_default: dict[int, Context] = {}


def default_context(device: int = 0) -> Context:
    ctx = _default.get(device)
    if ctx is None:
        ctx = _default[device] = Context(device)
    return ctx


def _is_torch(a) -> bool:
    return type(a).__module__.startswith("torch")


def _type_of(a) -> str:
    if _is_torch(a):
        t = _TORCH_NAME.get(str(a.dtype).replace("torch.", ""))
    else:
        t = next((k for k, d in _NP.items() if a.dtype == np.dtype(d)), None)
    if t is None:
        raise TypeError(f"{a.dtype} is not one of the ten sortable types")
    return t


def _host_ptr(a: np.ndarray) -> int:
    if not a.flags.c_contiguous:
        raise ValueError("the slice must be contiguous")
    if not a.flags.writeable:
        raise ValueError("the slice must be writeable")
    return a.ctypes.data


def _dev(a) -> bool:
    if _is_torch(a):
        if not a.is_cuda:
            raise ValueError("torch tensors must be on a CUDA device; pass numpy arrays for host slices")
        if not a.is_contiguous():
            raise ValueError("the slice must be contiguous")
        return True
    return False


def sort(a, ctx: Context | None = None) -> None:
    """Sort `a` in place, ascending in the crate's key order (src/lib.rs:99)."""
    ctx = ctx or default_context(a.device.index if _is_torch(a) else 0)
    t = _type_of(a)
    if _dev(a):
        ctx._check(getattr(lib(), f"ts_sort_dev_{t}")(ctx.handle, a.data_ptr(), a.numel()))
    else:
        ctx._check(getattr(lib(), f"ts_sort_{t}")(ctx.handle, _host_ptr(a), a.size))


def sort_with_buffer(a, buf, ctx: Context | None = None) -> None:
    """Sort with a caller-provided buffer of at least len(a) (src/lib.rs:122).
    Raises ValueError("buffer too small: need N, got M") like the crate's panic."""
    ctx = ctx or default_context(a.device.index if _is_torch(a) else 0)
    t = _type_of(a)
    if _type_of(buf) != t:
        raise TypeError("the buffer's type differs from the slice's")
    if _dev(a):
        if not _dev(buf):
            raise ValueError("a device slice needs a device buffer")
        ctx._check(getattr(lib(), f"ts_sort_dev_with_buffer_{t}")(ctx.handle, a.data_ptr(), a.numel(),
                                                                   buf.data_ptr(), buf.numel()))
    else:
        ctx._check(getattr(lib(), f"ts_sort_with_buffer_{t}")(ctx.handle, _host_ptr(a), a.size,
                                                               buf.ctypes.data, buf.size))


def sort_parallel(a, ctx: Context | None = None) -> None:
    """The crate's multi-core sort (src/lib.rs:224): the same device sort here."""
    ctx = ctx or default_context(a.device.index if _is_torch(a) else 0)
    t = _type_of(a)
    if _dev(a):
        ctx._check(getattr(lib(), f"ts_sort_dev_{t}")(ctx.handle, a.data_ptr(), a.numel()))
    else:
        ctx._check(getattr(lib(), f"ts_sort_parallel_{t}")(ctx.handle, _host_ptr(a), a.size))


def keys_order(keys, ctx: Context | None = None, out=None):
    """The stable order of `keys` (one sortable key per element): out[i] is the
    source index of output slot i (SortByKeyBuffer::order, src/by_key.rs:108)."""
    ctx = ctx or default_context(keys.device.index if _is_torch(keys) else 0)
    t = _type_of(keys)
    if _dev(keys):
        import torch

        if out is None:
            out = torch.empty(keys.numel(), dtype=torch.int32, device=keys.device)
        ctx._check(getattr(lib(), f"ts_sort_keys_order_dev_{t}")(ctx.handle, keys.data_ptr(), keys.numel(),
                                                                  out.data_ptr()))
        return out
    k = np.ascontiguousarray(keys)
    if out is None:
        out = np.empty(k.size, dtype=np.uint32)
    ctx._check(getattr(lib(), f"ts_sort_keys_order_{t}")(ctx.handle, k.ctypes.data, k.size, out.ctypes.data))
    return out


def apply_order(data, order, ctx: Context | None = None) -> None:
    """Put `data` in `order` in place: position i gets the element at order[i]."""
    ctx = ctx or default_context(data.device.index if _is_torch(data) else 0)
    if _is_torch(data):
        _dev(data)
        n = data.shape[0] if data.dim() else 0
        elem = data.element_size() * (data[0].numel() if n else 1)
        ctx._check(lib().ts_apply_order_dev(ctx.handle, data.data_ptr(), n, elem, order.data_ptr(), order.numel()))
        return
    n = data.shape[0] if data.ndim else 0
    elem = data.itemsize * (int(np.prod(data.shape[1:])) if data.ndim > 1 else 1)
    o = np.ascontiguousarray(order, dtype=np.uint32)
    ctx._check(lib().ts_apply_order(ctx.handle, _host_ptr(data), n, elem, o.ctypes.data, o.size))


def sort_segments(data, offsets, ctx: Context | None = None) -> None:
    """Sort every segment data[offsets[i]:offsets[i+1]] in place, independently
    (the crate's sort applied to each slice), in one device launch. `offsets`
    holds n_seg + 1 non-decreasing entries (numpy uint64 for host data, a CUDA
    int64 tensor for device data)."""
    ctx = ctx or default_context(data.device.index if _is_torch(data) else 0)
    t = _type_of(data)
    if _dev(data):
        n_seg = offsets.numel() - 1
        ctx._check(getattr(lib(), f"ts_sort_segments_dev_{t}")(ctx.handle, data.data_ptr(), data.numel(),
                                                                offsets.data_ptr(), max(n_seg, 0)))
        return
    o = np.ascontiguousarray(offsets, dtype=np.uint64)
    ctx._check(getattr(lib(), f"ts_sort_segments_{t}")(ctx.handle, _host_ptr(data), data.size, o.ctypes.data,
                                                        max(o.size - 1, 0)))


def segments_methods(key_bytes: int, ctx: Context | None = None, methods=None) -> list[int]:
    """Read (or set) the on-chip method of each segment length bin for keys of
    `key_bytes`: 0 bitonic, 1 radix with 4-bit digits, 2 radix with 8-bit digits,
    3 one MSD pass in shared memory, 4 (first bin only) one warp a segment, 5 (second bin,
    keys of up to 4 bytes) one warp a segment, 16 or 32 keys a lane, 6 (third and fourth
    bins, 4- and 8-byte keys) the MSD pass by thread groups, several segments a CTA."""
    ctx = ctx or default_context(0)
    arr = (ctypes.c_int * 4)(*(methods or [0, 0, 0, 0]))
    ctx._check(lib().ts_segments_methods(ctx.handle, key_bytes, arr, 1 if methods is not None else 0))
    return list(arr)


def segments_autotune(key_bytes: int, ctx: Context | None = None) -> list[int]:
    """Time each method on synthetic batches of every length bin on this GPU
    and keep the fastest; returns the chosen methods."""
    ctx = ctx or default_context(0)
    ctx._check(lib().ts_segments_autotune(ctx.handle, key_bytes))
    return segments_methods(key_bytes, ctx)


def learned_params(**overrides) -> LearnedParams:
    """The defaults of ts_learned_defaults with the given fields replaced."""
    p = LearnedParams()
    lib().ts_learned_defaults(ctypes.byref(p))
    for k, v in overrides.items():
        if not hasattr(p, k):
            raise TypeError(f"no learned-sort parameter {k!r}")
        setattr(p, k, v)
    return p


def sort_learned(a, params: LearnedParams | None = None, ctx: Context | None = None, **overrides) -> dict:
    """Sort `a` in place through the learned partition (same output as
    `sort`); returns the run's statistics (imbalance, training loss, whether it
    fell back to the plain sort, per-phase milliseconds)."""
    ctx = ctx or default_context(a.device.index if _is_torch(a) else 0)
    t = _type_of(a)
    if t not in LEARNED_TYPES:
        raise TypeError(f"the learned sort takes {', '.join(LEARNED_TYPES)} keys, not {t}")
    p = params if params is not None else learned_params(**overrides)
    st = LearnedStats()
    if _dev(a):
        ctx._check(getattr(lib(), f"ts_sort_learned_dev_{t}")(ctx.handle, a.data_ptr(), a.numel(), ctypes.byref(p),
                                                              ctypes.byref(st)))
    else:
        ctx._check(getattr(lib(), f"ts_sort_learned_{t}")(ctx.handle, _host_ptr(a), a.size, ctypes.byref(p),
                                                          ctypes.byref(st)))
    return st.as_dict()


LM_PIECES = 8  # pieces of every leaf's linear CDF


def lm_gradients(t, y, first, last, bp, y0, h, v, ctx: Context | None = None):
    """The learned leaves' backward kernel on CUDA tensors: returns (dL/dv, L)
    for L = mean_i (y0[j] + h[j] * PL_j(t_i) - y_i)^2, leaf j owning samples
    first[j]..last[j]; bp is [leaves, 7] (interior breakpoints), v is
    [leaves, 9] (heights); the gradient has v's shape."""
    import torch
    ctx = ctx or default_context(t.device.index)
    leaves = y0.numel()
    grad = torch.empty((leaves, LM_PIECES + 1), dtype=torch.float32, device=t.device)
    loss = ctypes.c_double(0.0)
    ctx._check(lib().ts_lm_gradients(ctx.handle, t.data_ptr(), y.data_ptr(), t.numel(), leaves, first.data_ptr(),
                                     last.data_ptr(), bp.data_ptr(), y0.data_ptr(), h.data_ptr(), v.data_ptr(),
                                     grad.data_ptr(), ctypes.byref(loss)))
    return grad, loss.value


def _key_array(items, key, dtype):
    vals = [key(x) for x in items]  # exactly one call per element (src/lib.rs:165-166)
    if dtype is None:
        if vals and isinstance(vals[0], np.generic):
            dtype = vals[0].dtype
        elif vals and isinstance(vals[0], float):
            dtype = np.float64
        else:
            dtype = np.int64
    return np.asarray(vals, dtype=dtype)


class SortByKeyBuffer:
    """Reusable memory for sort_by_key_with_buffer (src/by_key.rs:51-145):
    the device scratch of its own context, and the order of the last sort."""

    def __init__(self, capacity: int = 0, key_bytes: int = 8, device: int = 0):
        self.ctx = Context(device)
        self._order = np.empty(0, dtype=np.uint32)
        if capacity:
            self.ctx.reserve(capacity, key_bytes, with_order=True)

    def capacity(self, key_bytes: int = 8) -> int:
        return self.ctx.capacity(key_bytes, with_order=True)

    def order(self) -> np.ndarray:
        """After a sort, position i of the sorted slice holds the element that
        was at order()[i]. Empty before the first sort (src/by_key.rs:92-110)."""
        return self._order

    def apply_order(self, other, scratch=None) -> None:
        """Put `other` in the order of the last sort (src/by_key.rs:136-144).
        Raises ValueError on a length mismatch, as the crate panics."""
        n = len(other)
        if n != self._order.size:
            raise ValueError("apply_order: the slice's length differs from the last sorted slice's")
        if isinstance(other, np.ndarray) and other.dtype != object:
            apply_order(other, self._order, self.ctx)
        else:
            moved = [other[int(i)] for i in self._order]
            other[:] = moved
        if scratch is not None:
            scratch.clear()


def sort_by_key_with_buffer(items, buffer: SortByKeyBuffer, key, dtype=None) -> None:
    """Stable sort of `items` by key(x) (src/lib.rs:196, src/by_key.rs:175-235).
    `items` is a list or a numpy array; key runs once per element on the host."""
    keys = _key_array(items, key, dtype)
    n = keys.size
    if n < 2:
        buffer._order = np.arange(n, dtype=np.uint32)
        return
    if n > 0xFFFFFFFF:
        buffer._order = np.empty(0, dtype=np.uint32)  # order() is empty (src/by_key.rs:190-194)
        idx = np.argsort(keys, kind="stable")
        moved = [items[int(i)] for i in idx]
        items[:] = moved
        return
    buffer._order = keys_order(keys, buffer.ctx)
    buffer.apply_order(items)


def sort_by_key(items, key, dtype=None) -> None:
    """Stable sort by key, with a fresh buffer (src/lib.rs:152)."""
    sort_by_key_with_buffer(items, SortByKeyBuffer(), key, dtype)
