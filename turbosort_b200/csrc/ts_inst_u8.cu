// Instantiates the device sorts for 8-bit keys: unsigned, signed and (for
// 32/64 bits) IEEE float transforms.
#include "ts_engine.cuh"

namespace ts {
template ts_status sort_keys_device<uint8_t, 0>(ts_ctx*, uint8_t*, size_t, uint8_t*);
template ts_status sort_keys_device<uint8_t, 1>(ts_ctx*, uint8_t*, size_t, uint8_t*);
template ts_status order_device<uint8_t, 0>(ts_ctx*, const uint8_t*, size_t, uint32_t*);
template ts_status order_device<uint8_t, 1>(ts_ctx*, const uint8_t*, size_t, uint32_t*);
}  // namespace ts
