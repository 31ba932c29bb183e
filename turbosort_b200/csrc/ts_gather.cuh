// ts_gather.cuh — apply_order / move_into_order on the device
// (src/by_key.rs:136-144, :315-334): out[i] = in[order[i]] for elements of
// any size, moved as 16-, 8-, 4- or 1-byte words. Consecutive threads take
// consecutive words of the output, so writes coalesce and each element's
// words are read together.
#pragma once

#include "ts_common.cuh"

namespace ts {

template <typename W>
__global__ void __launch_bounds__(256) k_gather(const W* __restrict__ in, W* __restrict__ out,
                                                const uint32_t* __restrict__ order, size_t n, uint32_t wpe,
                                                uint32_t* __restrict__ error) {
    const size_t total = n * wpe;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x; g < total; g += stride) {
        size_t i = g, w = 0;
        if (wpe != 1) {
            i = g / wpe;
            w = g - i * wpe;
        }
        const uint32_t src = __ldg(order + i);
        if (src < n) {
            out[g] = in[(size_t)src * wpe + w];
        } else {
            atomicOr(error, ERR_BOUNDS);
        }
    }
}

}  // namespace ts
