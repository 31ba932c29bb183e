// ts_widths.cuh — the plain LSD at digit widths other than 8 bits.
//
// The crate sorts with byte digits, and 8-byte keys of at least 65,536 with
// 11-bit digits in six passes when its scatter does not stream
// (src/radix/mod.rs:43-54, :518-600). Here the width is a per-context choice
// per key width and length bin (ts_lsd_digit_bits, or the autotuner), from 4
// to 11 bits, for keys-only sorts below 2^31 keys. The kernels are the 8-bit
// sort's, instantiated at the other width: wider digits mean fewer passes but
// 16 x 2^bits per-warp counters in shared memory, so smaller tiles (and one
// CTA an SM at 10 bits for 8-byte keys and at 11 bits), and 2^bits look-back
// entries per tile. These sorts never divert.
#pragma once

#include "ts_engine.cuh"

namespace ts {

template <typename U, int XF, int B>
static ts_status run_lsd_width(ts_ctx* c, U* d_data, U* d_alt, size_t n, Plan** plan) {
    return run_lsd<U, XF, false, LsdCfg<U, false, 0, B>>(c, d_data, d_alt, d_data, nullptr, nullptr, nullptr, n, 1,
                                                          plan);
}

template <typename U, int XF>
ts_status run_lsd_bits(ts_ctx* c, int bits, U* d_data, U* d_alt, size_t n, Plan** plan) {
    switch (bits) {
        case 4: return run_lsd_width<U, XF, 4>(c, d_data, d_alt, n, plan);
        case 5: return run_lsd_width<U, XF, 5>(c, d_data, d_alt, n, plan);
        case 6: return run_lsd_width<U, XF, 6>(c, d_data, d_alt, n, plan);
        case 7: return run_lsd_width<U, XF, 7>(c, d_data, d_alt, n, plan);
        case 9: return run_lsd_width<U, XF, 9>(c, d_data, d_alt, n, plan);
        case 10: return run_lsd_width<U, XF, 10>(c, d_data, d_alt, n, plan);
        case 11: return run_lsd_width<U, XF, 11>(c, d_data, d_alt, n, plan);
    }
    return fail(c, TS_ERR_INTERNAL, "digit width");
}

}  // namespace ts
