// ts_gather.cuh — apply_order / move_into_order on the device
// (src/by_key.rs:136-144, :315-334): out[i] = in[order[i]] for elements of
// any size, moved as 16-, 8-, 4- or 1-byte words. Consecutive threads take
// consecutive words of the output, so writes coalesce and each element's
// words are read together.
#pragma once

#include "ts_common.cuh"

namespace ts {

// Each thread moves GATHER_ILP words per round, their loads issued together:
// the reads are random, so the number in flight sets the speed.
constexpr int GATHER_ILP = 4;

template <typename W>
__global__ void __launch_bounds__(256) k_gather(const W* __restrict__ in, W* __restrict__ out,
                                                const uint32_t* __restrict__ order, size_t n, size_t n_src,
                                                uint32_t wpe, uint32_t* __restrict__ error) {
    const size_t total = n * wpe;
    const size_t step = (size_t)gridDim.x * blockDim.x * GATHER_ILP;
    for (size_t base = (size_t)blockIdx.x * blockDim.x * GATHER_ILP + threadIdx.x; base < total; base += step) {
        uint32_t src[GATHER_ILP];
        size_t w[GATHER_ILP];
#pragma unroll
        for (int e = 0; e < GATHER_ILP; ++e) {
            const size_t g = base + (size_t)e * blockDim.x;
            size_t i = g;
            w[e] = 0;
            if (wpe != 1) {
                i = g / wpe;
                w[e] = g - i * wpe;
            }
            src[e] = g < total ? __ldcs(order + i) : 0u;
        }
        W v[GATHER_ILP];
#pragma unroll
        for (int e = 0; e < GATHER_ILP; ++e) {
            const size_t g = base + (size_t)e * blockDim.x;
            if (g < total && src[e] < n_src) v[e] = in[(size_t)src[e] * wpe + w[e]];
        }
#pragma unroll
        for (int e = 0; e < GATHER_ILP; ++e) {
            const size_t g = base + (size_t)e * blockDim.x;
            if (g >= total) continue;
            if (src[e] < n_src) __stcs(out + g, v[e]);
            else atomicOr(error, ERR_BOUNDS);
        }
    }
}

}  // namespace ts
