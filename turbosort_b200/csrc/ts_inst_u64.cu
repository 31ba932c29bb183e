// Instantiates the device sorts for 64-bit keys: unsigned, signed and (for
// 32/64 bits) IEEE float transforms.
#include "ts_engine.cuh"
#include "ts_pipeline.cuh"

namespace ts {
template ts_status sort_keys_device<uint64_t, 0>(ts_ctx*, uint64_t*, size_t, uint64_t*);
template ts_status sort_keys_device<uint64_t, 1>(ts_ctx*, uint64_t*, size_t, uint64_t*);
template ts_status order_device<uint64_t, 0>(ts_ctx*, const uint64_t*, size_t, uint32_t*);
template ts_status order_device<uint64_t, 1>(ts_ctx*, const uint64_t*, size_t, uint32_t*);
template ts_status sort_keys_device<uint64_t, 2>(ts_ctx*, uint64_t*, size_t, uint64_t*);
template ts_status order_device<uint64_t, 2>(ts_ctx*, const uint64_t*, size_t, uint32_t*);
template ts_status pipeline_sort<uint64_t, 0>(ts_ctx*, uint64_t*, size_t);
template ts_status pipeline_sort<uint64_t, 1>(ts_ctx*, uint64_t*, size_t);
template ts_status pipeline_sort<uint64_t, 2>(ts_ctx*, uint64_t*, size_t);
template ts_status pipeline_order<uint64_t, 0>(ts_ctx*, const uint64_t*, size_t, uint32_t*);
template ts_status pipeline_order<uint64_t, 1>(ts_ctx*, const uint64_t*, size_t, uint32_t*);
template ts_status pipeline_order<uint64_t, 2>(ts_ctx*, const uint64_t*, size_t, uint32_t*);
}  // namespace ts
