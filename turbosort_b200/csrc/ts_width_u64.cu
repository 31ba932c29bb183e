// Instantiates the plain LSD of 64-bit keys at digit widths other than 8
// (unsigned, signed and IEEE float transforms).
#include "ts_widths.cuh"

namespace ts {
template ts_status run_lsd_bits<uint64_t, 0>(ts_ctx*, int, uint64_t*, uint64_t*, size_t, Plan**);
template ts_status run_lsd_bits<uint64_t, 1>(ts_ctx*, int, uint64_t*, uint64_t*, size_t, Plan**);
template ts_status run_lsd_bits<uint64_t, 2>(ts_ctx*, int, uint64_t*, uint64_t*, size_t, Plan**);
}  // namespace ts
