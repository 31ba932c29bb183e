// ts_small.cuh — the short-slice tiers and the one-byte counting sort.
//
//   k_warp_sort    one warp sorts up to 32 or WARP_TIER_MAX keys in registers
//                  (bitonic: shuffles between lanes, swaps inside a lane)
//   k_small_sort   one CTA sorts up to SMALL_MAX keys with a bitonic network
//                  in shared memory, padding with the largest key exactly as
//                  the crate's AVX2 networks pad with u32::MAX
//                  (src/arch/x86_64/avx2.rs:311-313, :566-584; src/tiny.rs:15,
//                  src/small.rs:11). With positions it compares (key, pos),
//                  which makes it stable for sort_by_key (src/by_key.rs:239-249).
//   k_count8/k_fill8  counting sort of one-byte keys
//                  (src/radix/mod.rs:123-164): one read to count, one write
//                  that fills each digit's run.
#pragma once

#include "ts_common.cuh"

namespace ts {

constexpr int SMALL_MAX = 4096;
constexpr int WARP_TIER_MAX = 256;  // k_warp_sort with 8 keys a lane
constexpr int SMALL_THREADS = 1024;

// `in` and `out` may be the same array (the keys are all in shared memory
// before the first write), so neither is declared restrict.
template <typename U, int XF, bool PAIRS>
__global__ void __launch_bounds__(SMALL_THREADS) k_small_sort(const U* in, U* out, uint32_t* __restrict__ order, int n,
                                                              int write_keys) {
    __shared__ U sk[SMALL_MAX];
    __shared__ uint32_t sv[PAIRS ? SMALL_MAX : 1];
    int p2 = 1;
    while (p2 < n) p2 <<= 1;
    for (int i = threadIdx.x; i < p2; i += blockDim.x) {
        sk[i] = i < n ? to_key<U, XF>(in[i]) : (U)~(U)0;
        if constexpr (PAIRS) sv[i] = i < n ? (uint32_t)i : 0xffffffffu;
    }
    __syncthreads();
    for (int k = 2; k <= p2; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < p2; i += blockDim.x) {
                const int ixj = i ^ j;
                if (ixj > i) {
                    const bool up = (i & k) == 0;
                    const U a = sk[i], b = sk[ixj];
                    bool gt;
                    if constexpr (PAIRS) gt = a > b || (a == b && sv[i] > sv[ixj]);
                    else gt = a > b;
                    if (gt == up) {
                        sk[i] = b;
                        sk[ixj] = a;
                        if constexpr (PAIRS) {
                            const uint32_t t = sv[i];
                            sv[i] = sv[ixj];
                            sv[ixj] = t;
                        }
                    }
                }
            }
            __syncthreads();
        }
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        if (write_keys) out[i] = from_key<U, XF>(sk[i]);
        if constexpr (PAIRS) order[i] = sv[i];
    }
}

// One warp sorts up to 32 * R keys in registers (warp_bitonic; k_warp_sort is
// its launch for one slice): element e = r * 32 + lane
// sits in register r of that lane. A bitonic network over the next power of
// two, padded with the largest key as the crate's AVX2 tiers pad
// (src/arch/x86_64/avx2.rs:211-313): partners 32 and more apart are in the
// same lane (a register swap), closer ones in another lane (a shuffle). No
// shared memory and no block barrier: the tier for the slices the crate
// sends to its register networks (src/tiny.rs:15, src/small.rs:11).
template <typename U, int XF, int R>
__device__ __forceinline__ void warp_bitonic(const U* in, U* out, int n, int lane) {
    constexpr int N = 32 * R;
    U v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int e = r * 32 + lane;
        v[r] = e < n ? to_key<U, XF>(in[e]) : (U)~(U)0;
    }
#pragma unroll
    for (int k = 2; k <= N; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            if (j >= 32) {
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const int rp = r ^ (j >> 5);
                    if (rp > r) {
                        const bool up = ((r * 32) & k) == 0;
                        const U a = v[r], b = v[rp];
                        const bool sw = (a > b) == up;
                        v[r] = sw ? b : a;
                        v[rp] = sw ? a : b;
                    }
                }
            } else {
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const int e = r * 32 + lane;
                    const U o = __shfl_xor_sync(0xffffffffu, v[r], j);
                    const bool up = (e & k) == 0;
                    const bool lower = (e & j) == 0;
                    const bool keep_min = lower == up;
                    v[r] = keep_min ? (o < v[r] ? o : v[r]) : (o > v[r] ? o : v[r]);
                }
            }
        }
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int e = r * 32 + lane;
        if (e < n) out[e] = from_key<U, XF>(v[r]);
    }
}

template <typename U, int XF, int R>
__global__ void __launch_bounds__(32) k_warp_sort(U* d, int n) {
    warp_bitonic<U, XF, R>(d, d, n, threadIdx.x);
}

template <int XF>
__global__ void __launch_bounds__(512) k_count8(const uint8_t* __restrict__ src, size_t n,
                                                unsigned long long* __restrict__ ghist) {
    constexpr int COPIES = 8;
    __shared__ uint32_t h[256 * COPIES];
    for (int i = threadIdx.x; i < 256 * COPIES; i += blockDim.x) h[i] = 0;
    __syncthreads();
    const int copy = threadIdx.x % COPIES;
    const size_t nv = n / 16;
    const uint4* v = reinterpret_cast<const uint4*>(src);
    const bool vec_ok = ((uintptr_t)src & 15) == 0;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    if (vec_ok) {
        for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += stride) {
            union {
                uint4 q;
                uint8_t b[16];
            } x;
            x.q = __ldcs(v + i);
#pragma unroll
            for (int e = 0; e < 16; ++e) atomicAdd(&h[(uint32_t)to_key<uint8_t, XF>(x.b[e]) * COPIES + copy], 1u);
        }
    }
    for (size_t i = (vec_ok ? nv * 16 : 0) + (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        atomicAdd(&h[(uint32_t)to_key<uint8_t, XF>(src[i]) * COPIES + copy], 1u);
    __syncthreads();
    for (int d = threadIdx.x; d < 256; d += blockDim.x) {
        uint32_t s = 0;
#pragma unroll
        for (int c = 0; c < COPIES; ++c) s += h[d * COPIES + c];
        if (s) atomicAdd(&ghist[d], (unsigned long long)s);
    }
}

// Each thread writes 16 consecutive bytes; the digit of each output slot is
// the first digit whose inclusive count exceeds the slot.
template <int XF>
__global__ void __launch_bounds__(256) k_fill8(uint8_t* __restrict__ dst, size_t n,
                                               const unsigned long long* __restrict__ ghist) {
    __shared__ unsigned long long incl[256];
    if (threadIdx.x < 32) {
        unsigned long long carry = 0;
        for (int r0 = 0; r0 < 256; r0 += 32) {
            const int lane = threadIdx.x;
            unsigned long long x = ghist[r0 + lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            incl[r0 + lane] = carry + x;
            carry += __shfl_sync(0xffffffffu, x, 31);
        }
    }
    __syncthreads();
    const size_t stride = (size_t)gridDim.x * blockDim.x * 16;
    const bool vec_ok = ((uintptr_t)dst & 15) == 0;
    for (size_t b = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) * 16; b < n; b += stride) {
        int lo = 0, hi = 255;  // first digit with incl > b
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (incl[mid] > b) hi = mid;
            else lo = mid + 1;
        }
        int d = lo;
        union {
            uint4 q;
            uint8_t e[16];
        } x;
#pragma unroll
        for (int e = 0; e < 16; ++e) {
            while (d < 255 && incl[d] <= b + e) ++d;
            x.e[e] = from_key<uint8_t, XF>((uint8_t)d);
        }
        if (vec_ok && b + 16 <= n) {
            *reinterpret_cast<uint4*>(dst + b) = x.q;
        } else {
            for (int e = 0; e < 16 && b + e < n; ++e) dst[b + e] = x.e[e];
        }
    }
}

}  // namespace ts
