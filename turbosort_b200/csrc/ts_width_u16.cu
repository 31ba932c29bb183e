// Instantiates the plain LSD of 16-bit keys at digit widths other than 8
// (unsigned, signed transforms).
#include "ts_widths.cuh"

namespace ts {
template ts_status run_lsd_bits<uint16_t, 0>(ts_ctx*, int, uint16_t*, uint16_t*, size_t, Plan**);
template ts_status run_lsd_bits<uint16_t, 1>(ts_ctx*, int, uint16_t*, uint16_t*, size_t, Plan**);
}  // namespace ts
