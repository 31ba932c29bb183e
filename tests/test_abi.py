"""The C ABI library loads and exports every symbol include/turbosort.h
declares (no GPU needed: nothing here calls into the device)."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TYPES = ("u8", "u16", "u32", "u64", "i8", "i16", "i32", "i64", "f32", "f64")


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "turbosort.h")).read()
    names = set(re.findall(r"\b(ts_[a-z0-9_]+)\s*\(", text))
    macro = re.search(r"#define TS_DECLARE_SORTS\(SUF, T\)(.*?)\n\n", text, re.S).group(1)
    per_type = set(re.findall(r"\b(ts_[a-z0-9_]+)##SUF\b", macro))
    names = {n for n in names if not n.endswith("_")}
    for stem in per_type:
        for t in TYPES:
            names.add(stem + t)
    return sorted(names)


def test_header_declares_the_crate_surface():
    names = declared_symbols()
    for t in TYPES:
        for stem in ("ts_sort_", "ts_sort_with_buffer_", "ts_sort_parallel_", "ts_sort_keys_order_",
                     "ts_sort_dev_"):
            assert stem + t in names
    assert "ts_apply_order" in names and "ts_ctx_create" in names


def test_library_exports_every_declared_symbol():
    import turbosort_b200 as ts

    L = ts.lib()
    missing = [n for n in declared_symbols() if not hasattr(L, n)]
    assert not missing, missing


def test_status_strings_and_no_device_path():
    import turbosort_b200 as ts

    L = ts.lib()
    assert L.ts_status_str(1) == b"buffer too small"
    assert L.ts_status_str(2) == b"length mismatch"
    # null context is rejected without touching a device
    assert L.ts_sort_u32(None, None, 0) == 6
