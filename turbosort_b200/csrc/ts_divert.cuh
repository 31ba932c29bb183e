// ts_divert.cuh — finishing the runs a diverted sort leaves
// (src/radix/divert.rs:60-81).
//
// When k_plan diverts, the passes sort only the digits from divert_shift up:
// the keys then come out ordered by that prefix, in runs of keys sharing it
// (most runs one key long), and each run only needs sorting within itself.
//   k_divert_runs  one read of the keys, 32 consecutive keys a warp: a key
//                  whose prefix differs from its predecessor's and equals its
//                  successor's starts a run of two or more. Its thread finds
//                  the run's end (galloping, then bisecting, over the sorted
//                  prefixes), sorts a run of up to DIVERT_SHORT keys itself
//                  (insertion sort, as divert.rs:85-92 does up to SHORT_RUN),
//                  and lists the start of a longer one.
//   k_divert_long  one CTA per listed run: the segmented sort's on-chip MSD
//                  routine (msd_sort), or its CTA-level LSD through the free
//                  ping-pong buffer for runs beyond shared memory.
// Runs are disjoint and a permutation inside a run changes no prefix, so
// threads that read neighbouring keys while another thread rewrites a run
// still see the right prefixes. Both kernels are no-ops unless the plan
// diverted. The output equals the full sort's: runs are in prefix order, and
// each run is sorted by its whole key.
#pragma once

#include "ts_common.cuh"
#include "ts_segmented.cuh"

namespace ts {

constexpr int DIVERT_SHORT = 16;  // src/radix/divert.rs:23

// The end of the run that starts at s, in keys sorted by their prefix
// p = to_key(key) >> shift; d[s + 1] is known to share it.
template <typename U, int XF>
__device__ size_t divert_run_end(const U* d, size_t n, size_t s, int shift) {
    const unsigned long long p = (unsigned long long)to_key<U, XF>(d[s]) >> shift;
    auto same = [&](size_t i) { return ((unsigned long long)to_key<U, XF>(d[i]) >> shift) == p; };
    size_t lo = s + 1;  // shares the prefix
    size_t step = 1;
    size_t hi = n;      // first index known not to share it (or n)
    while (true) {
        const size_t probe = lo + step;
        if (probe >= n) break;
        if (!same(probe)) {
            hi = probe;
            break;
        }
        lo = probe;
        step <<= 1;
    }
    while (hi - lo > 1) {
        const size_t mid = lo + (hi - lo) / 2;
        if (same(mid)) lo = mid;
        else hi = mid;
    }
    return hi;
}

template <typename U, int XF>
__global__ void __launch_bounds__(256) k_divert_runs(const Plan* __restrict__ plan, U* d, size_t n,
                                                     unsigned long long* __restrict__ runs,
                                                     unsigned long long* __restrict__ n_runs, size_t runs_cap,
                                                     uint32_t* __restrict__ error) {
    if (plan->mode != MODE_SORT || plan->divert_shift <= 0) return;
    const int shift = plan->divert_shift;
    auto pre = [&](U v) { return (unsigned long long)to_key<U, XF>(v) >> shift; };
    const int lane = threadIdx.x & 31;
    const size_t gw = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
    for (size_t wb = gw * 32; wb < n; wb += nw * 32) {  // warp-uniform
        const size_t i = wb + lane;
        const bool valid = i < n;
        const U v = valid ? d[i] : (U)0;
        U prev = __shfl_up_sync(0xffffffffu, v, 1);
        U next = __shfl_down_sync(0xffffffffu, v, 1);
        if (lane == 0 && valid && i > 0) prev = d[i - 1];
        if (lane == 31 && i + 1 < n) next = d[i + 1];
        if (!valid) continue;
        const unsigned long long p = pre(v);
        const bool start = i == 0 || pre(prev) != p;
        if (!start || i + 1 >= n || pre(next) != p) continue;
        // a run of two or more keys starts here
        const size_t e = divert_run_end<U, XF>(d, n, i, shift);
        const size_t len = e - i;
        if (len <= (size_t)DIVERT_SHORT) {
            U k[DIVERT_SHORT];
            for (size_t j = 0; j < len; ++j) k[j] = to_key<U, XF>(d[i + j]);
            bool moved = false;
            for (size_t j = 1; j < len; ++j) {
                const U x = k[j];
                size_t q = j;
                while (q > 0 && k[q - 1] > x) {
                    k[q] = k[q - 1];
                    --q;
                }
                k[q] = x;
                moved |= q != j;
            }
            if (moved)
                for (size_t j = 0; j < len; ++j) d[i + j] = from_key<U, XF>(k[j]);
        } else {
            const unsigned long long slot = atomicAdd(n_runs, 1ull);
            if (slot < runs_cap) runs[slot] = i;
            else atomicOr(error, ERR_BOUNDS);  // cannot happen: a listed run holds more than DIVERT_SHORT keys
        }
    }
}

template <typename U, int XF>
__global__ void __launch_bounds__(SEG_THREADS, 1)
    k_divert_long(const Plan* __restrict__ plan, U* d, U* __restrict__ alt, size_t n,
                  const unsigned long long* __restrict__ runs, const unsigned long long* __restrict__ n_runs,
                  unsigned int* __restrict__ counter, uint32_t* __restrict__ error) {
    if (plan->mode != MODE_SORT || plan->divert_shift <= 0) return;
    extern __shared__ __align__(128) unsigned char smem[];
    // the last 16 bytes of the launch's shared memory, which msd_sort leaves alone
    unsigned long long* item_s = reinterpret_cast<unsigned long long*>(smem + MSD_SMEM - 16);
    const int shift = plan->divert_shift;
    const unsigned long long total = *n_runs;
    for (;;) {
        if (threadIdx.x == 0) {
            const unsigned long long item = atomicAdd(counter, 1u);
            item_s[0] = item;
            if (item < total) {
                const size_t s = runs[item];
                item_s[1] = divert_run_end<U, XF>(d, n, s, shift) - s;
            }
        }
        __syncthreads();
        const unsigned long long item = item_s[0];
        if (item >= total) break;
        const size_t s = runs[item];
        const unsigned long long len = item_s[1];
        if (len <= 0x7fffffffull) {
            msd_sort<U, XF>(d + s, d + s, alt + s, (int)len, smem);
        } else if (threadIdx.x == 0) {
            atomicOr(error, ERR_BOUNDS);  // runs of 2^31 keys and more are beyond the CTA sort
        }
        __syncthreads();
    }
}

}  // namespace ts
