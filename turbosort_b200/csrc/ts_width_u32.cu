// Instantiates the plain LSD of 32-bit keys at digit widths other than 8
// (unsigned, signed and IEEE float transforms).
#include "ts_widths.cuh"

namespace ts {
template ts_status run_lsd_bits<uint32_t, 0>(ts_ctx*, int, uint32_t*, uint32_t*, size_t, Plan**);
template ts_status run_lsd_bits<uint32_t, 1>(ts_ctx*, int, uint32_t*, uint32_t*, size_t, Plan**);
template ts_status run_lsd_bits<uint32_t, 2>(ts_ctx*, int, uint32_t*, uint32_t*, size_t, Plan**);
}  // namespace ts
