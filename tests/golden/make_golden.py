"""Writes tests/golden/kat.json: known-answer vectors restated from the
turbosort crate's own tests and docs, plus a few derived by an independent
method (Rust's documented `total_cmp` formula, not the radix transform).

The crate is Rust and cannot be built here, so its tests cannot run; their
inputs and asserted outputs are written out below as data, each with the
file:line it comes from. Run: python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import math
import os
import struct

HERE = os.path.dirname(os.path.abspath(__file__))
M64 = (1 << 64) - 1


def xorshift64(state: int):
    """The crate's test generator (13/7/17), e.g. src/key.rs:256-262."""
    while True:
        state ^= (state << 13) & M64
        state ^= state >> 7
        state ^= (state << 17) & M64
        yield state


def f32_bits(x: float) -> int:
    return struct.unpack("<I", struct.pack("<f", x))[0]


def f64_bits(x: float) -> int:
    return struct.unpack("<Q", struct.pack("<d", x))[0]


def total_cmp_key32(b: int) -> int:
    """Rust std f32::total_cmp: i ^ (((i >> 31) as u32) >> 1), compared as i32."""
    i = b - (1 << 32) if b & 0x80000000 else b
    m = ((i >> 31) & 0xFFFFFFFF) >> 1
    v = (i ^ m) & 0xFFFFFFFF
    return v - (1 << 32) if v & 0x80000000 else v


def total_cmp_key64(b: int) -> int:
    i = b - (1 << 64) if b & (1 << 63) else b
    m = ((i >> 63) & M64) >> 1
    v = (i ^ m) & M64
    return v - (1 << 64) if v & (1 << 63) else v


F32_MIN_POS = 1.1754943508222875e-38
F32_MAX = 3.4028234663852886e38
NAN32 = 0x7FC00000  # f32::NAN: sign bit clear
NAN64 = 0x7FF8000000000000


def main() -> None:
    kat: dict = {}

    # src/key.rs:206-213 — i32 MIN < -1 < 0 < 1 < MAX keep strict key order.
    kat["key_order_i32"] = [-(2**31), -1, 0, 1, 2**31 - 1]
    # src/key.rs:216-235 — f32 -inf < -1 < -0 < +0 < 1 < inf < NaN.
    kat["key_order_f32_bits"] = [f32_bits(-math.inf), f32_bits(-1.0), 0x80000000, 0,
                                 f32_bits(1.0), f32_bits(math.inf), NAN32]

    # src/key.rs:253-282 — total_cmp order on edge and xorshift bit patterns.
    edges = [0, 1, 0x7FFFFFFF, 0x80000000, 0x80000001, 0xFFFFFFFF]
    f32s = list(edges)
    f64s = list(edges) + [1 << 63, M64]
    g = xorshift64(0x9E3779B97F4A7C15)
    for _ in range(2000):
        r = next(g)
        f32s.append(r & 0xFFFFFFFF)
        f64s.append(r)
    kat["total_cmp_f32"] = {"bits": f32s, "sorted": sorted(f32s, key=total_cmp_key32)}
    kat["total_cmp_f64"] = {"bits": f64s, "sorted": sorted(f64s, key=total_cmp_key64)}

    # tests/correctness.rs:249-281 — f32 edge cases and their asserted order.
    inp = [1.0, -1.0, 0.0, -0.0, math.inf, -math.inf, None, -F32_MAX, F32_MAX, F32_MIN_POS, -F32_MIN_POS]
    kat["float_edge_f32"] = {
        "input_bits": [NAN32 if x is None else f32_bits(x) for x in inp],
        "expected_bits": [f32_bits(-math.inf), f32_bits(-F32_MAX), f32_bits(-1.0), f32_bits(-F32_MIN_POS),
                          0x80000000, 0, f32_bits(F32_MIN_POS), f32_bits(1.0), f32_bits(F32_MAX),
                          f32_bits(math.inf), NAN32],
    }
    # tests/correctness.rs:283-303 — f64.
    kat["float_edge_f64"] = {
        "input_bits": [f64_bits(1.0), f64_bits(-1.0), 0, 1 << 63, f64_bits(math.inf), f64_bits(-math.inf), NAN64],
        "expected_bits": [f64_bits(-math.inf), f64_bits(-1.0), 1 << 63, 0, f64_bits(1.0), f64_bits(math.inf), NAN64],
    }
    # tests/correctness.rs:307-324 — signed extremes.
    kat["signed_edge"] = {
        "i32": {"input": [2**31 - 1, -(2**31), 0, -1, 1], "expected": [-(2**31), -1, 0, 1, 2**31 - 1]},
        "i64": {"input": [2**63 - 1, -(2**63), 0, -1, 1], "expected": [-(2**63), -1, 0, 1, 2**63 - 1]},
        "i8": {"input": [127, -128, 0, -1, 1], "expected": [-128, -1, 0, 1, 127]},
        "i16": {"input": [32767, -32768, 0, -1, 1], "expected": [-32768, -1, 0, 1, 32767]},
    }
    # src/lib.rs doc examples (:18-20, :26-29, :82-84, :92-96, :116-119).
    kat["doc_examples"] = [
        {"type": "u32", "input": [5, 3, 8, 1, 9, 2, 7, 4, 6], "expected": [1, 2, 3, 4, 5, 6, 7, 8, 9]},
        {"type": "u32", "input": [5, 3, 8, 1, 9], "expected": [1, 3, 5, 8, 9], "with_buffer": True},
        {"type": "i32", "input": [3, -1, 4, -1, 5, -9], "expected": [-9, -1, -1, 3, 4, 5]},
        {"type": "u64", "input": [42, 7, 99, 1, 0], "expected": [0, 1, 7, 42, 99], "with_buffer": True},
    ]
    # src/lib.rs:91-97 — NaN last, -0 before +0 (README.md:33-41 shows the same).
    kat["doc_f32_bits"] = {
        "input_bits": [f32_bits(1.0), NAN32, 0x80000000, 0, f32_bits(-math.inf)],
        "expected_bits": [f32_bits(-math.inf), 0x80000000, 0, f32_bits(1.0), NAN32],
    }
    # src/by_key.rs:101-107 — words by length, order() == [1, 0, 3, 2].
    kat["by_key_words"] = {"keys_u32": [4, 3, 5, 4], "order": [1, 0, 3, 2]}
    # README.md:63-66 — ids [30, 10, 20], order() == [1, 2, 0].
    kat["by_key_ids"] = {"keys_u32": [30, 10, 20], "order": [1, 2, 0]}
    # src/lib.rs:145-147 / README.md:53-55 — people by age, stable.
    kat["by_key_people_age"] = {"keys_u32": [31, 25, 31, 25], "order": [1, 3, 0, 2]}
    # README.md:57-60 — the sorted people again, by name length (5,4,3,5).
    kat["by_key_people_name_len"] = {"keys_u32": [5, 4, 3, 5], "order": [2, 1, 0, 3]}

    # src/radix/divert.rs:289 and :293-316 — digit-skipping arithmetic.
    kat["log2_eighths"] = [[1 << 20, 160]]
    n20, n16 = 1 << 20, 1 << 16
    kat["skippable_digits"] = [
        {"n_live": 8, "len": n20, "max": n20 // 256 + 64, "expect": 5},
        {"n_live": 4, "len": n16, "max": n16 // 256, "expect": 0},
        {"n_live": 4, "len": 1024, "max": 4, "expect": 0},
        {"n_live": 8, "len": 1024, "max": 4, "expect": 6},
        {"n_live": 8, "len": n16, "max": n16 - 1, "expect": 0},
        {"n_live": 0, "len": n16, "max": 1, "expect": 0},
        {"n_live": 3, "len": n16, "max": 1, "expect": 0},
    ]
    # src/radix/histogram.rs:138-147 — varying_bits masks.
    kat["varying_bits"] = {
        "u64_keys": [(0x1111222200004455 | ((i % 256) << 16) | ((i // 256) << 63)) & M64 for i in range(300)],
        "u64_expect": 0x80000000_00FF0000,
        "u32_sevens": [7] * 5,
        "u32_expect": 0,
        "u16_keys": [(i * 0x9E37) & 0xFFFF for i in range(300)],
        "u16_expect": None,
    }
    # src/radix/histogram.rs:150-158 — live passes [3, 4].
    kat["live_passes"] = {"keys_u64": [((i * 2654435761) % 4099) << 24 for i in range(10000)], "live": [3, 4]}

    # tests/correctness.proptest-regressions:7-8 — the two shrunk failing inputs.
    kat["regressions"] = {
        "f32": [0.0, 0.0, 0.0, -1.6976289, -1.5736036e31],
        "i32": [0, 0, 0, 0, 0, 0, 0, 0, 423439103, 0, -459012928, -1, -1, -1, 0, -1329394665, -1, 0, 0, 0, 0,
                -1329394665, 0, 0, 0, 162020954, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 423439104, 126044353, 0, 0, 0, 0,
                0, 0, -1, 0, 0, 0, 0, 0, 0, 0, 423439103, 423439103, 423439103, -1, 423439103, 0, 0, 0, 0, 0, 0,
                0, 0, 0, 0, 0, 0, 0, 0, -2, -843883178, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, -1, 0, 0, 0, 0, 0, 0, 0,
                0, 0, 0, -1, -1, 0, 0, 0, -1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0,
                0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, -1, 423439103, -1, 423439103, 423439103,
                -1, 423439103, -1, -1, -1, 0, -1, -1, -1, -1, -1, 0, -2],
    }

    with open(os.path.join(HERE, "kat.json"), "w") as f:
        json.dump(kat, f, indent=None, separators=(",", ":"))


if __name__ == "__main__":
    main()
