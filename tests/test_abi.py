"""The C ABI library loads and exports every symbol include/turbosort.h
declares (no GPU needed: nothing here calls into the device)."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TYPES = ("u8", "u16", "u32", "u64", "i8", "i16", "i32", "i64", "f32", "f64")


def declared_symbols():
    """Every function the header declares: plain declarations, plus each
    per-type macro (TS_DECLARE_*) expanded for the suffixes it is invoked with."""
    text = open(os.path.join(ROOT, "include", "turbosort.h")).read()
    names = {n for n in re.findall(r"\b(ts_[a-z0-9_]+)\s*\(", text) if not n.endswith("_")}
    for macro, body in re.findall(r"#define (TS_DECLARE_[A-Z]+)\(SUF, T\)(.*?)\n\n", text, re.S):
        stems = set(re.findall(r"\b(ts_[a-z0-9_]+)##SUF\b", body))
        suffixes = re.findall(r"^" + macro + r"\((\w+), \w+\)", text, re.M)
        assert stems and suffixes, macro
        for stem in stems:
            for t in suffixes:
                names.add(stem + t)
    return sorted(names)


def test_header_declares_the_crate_surface():
    names = declared_symbols()
    for t in TYPES:
        for stem in ("ts_sort_", "ts_sort_with_buffer_", "ts_sort_parallel_", "ts_sort_keys_order_",
                     "ts_sort_dev_"):
            assert stem + t in names
    assert "ts_apply_order" in names and "ts_ctx_create" in names
    for t in TYPES:
        assert "ts_sort_segments_" + t in names and "ts_sort_segments_dev_" + t in names
    for t in ("u32", "u64", "i32", "i64", "f32", "f64"):
        assert "ts_sort_learned_" + t in names and "ts_sort_learned_dev_" + t in names
    assert "ts_lm_gradients" in names and "ts_sort_dev_noalloc_u32" in names


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
    assert L.ts_ctx_transfer_pipeline(None, 8, 0) == 6
    assert L.ts_sort_keys_order_u64(None, None, 0, None) == 6
    assert L.ts_apply_order(None, None, 0, 16, None, 0) == 6
    assert L.ts_sort_segments_u32(None, None, 0, None, 0) == 6


def test_learned_structs_match_the_header():
    """The ctypes mirrors of ts_learned_params / ts_learned_stats have the C
    layout (sizes and every field offset, from a C program built with gcc)."""
    import subprocess
    import tempfile

    import turbosort_b200 as ts

    fields = {"ts_learned_params": ts.LearnedParams, "ts_learned_stats": ts.LearnedStats}
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "turbosort.h"', "int main(void) {"]
    for cname, cls in fields.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for f, _ in cls._fields_:
            lines.append(f'printf("{cname}.{f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("return 0; }")
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "layout.c"), os.path.join(d, "layout")
        open(src, "w").write("\n".join(lines))
        subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), src, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split("\n")
    got = dict(line.split() for line in out if line)
    for cname, cls in fields.items():
        assert int(got[cname]) == ctypes.sizeof(cls), cname
        for f, _ in cls._fields_:
            assert int(got[f"{cname}.{f}"]) == getattr(cls, f).offset, (cname, f)
