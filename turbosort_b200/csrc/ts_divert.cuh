// ts_divert.cuh — finishing the runs a diverted sort leaves
// (src/radix/divert.rs:60-81).
//
// When the plan diverts, the passes sort only the digits from divert_shift up:
// the keys then come out ordered by that prefix, in runs of keys sharing it
// (most runs one key long), and each run only needs sorting within itself.
//   k_divert_runs  one read of the keys, 16-byte loads, 32 * KPT consecutive
//                  keys a warp step: a key
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

// The run starting at s (len keys, 2 <= len <= DIVERT_SHORT) sorted in place.
template <typename U, int XF>
__device__ void divert_sort_short(U* d, size_t s, size_t len) {
    if (len == 2) {  // most runs: two keys, kept in registers
        const U a = d[s], b = d[s + 1];
        if (to_key<U, XF>(a) > to_key<U, XF>(b)) {
            d[s] = b;
            d[s + 1] = a;
        }
        return;
    }
    U k[DIVERT_SHORT];
    for (size_t j = 0; j < len; ++j) k[j] = to_key<U, XF>(d[s + j]);
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
        for (size_t j = 0; j < len; ++j) d[s + j] = from_key<U, XF>(k[j]);
}

// A run of three or more keys starting at i: its end, then a sort by this
// thread or a place in the list. Rare, so kept out of the streaming loop.
template <typename U, int XF>
__device__ __noinline__ void divert_long_run(U* d, size_t n, size_t i, int shift, unsigned long long* runs,
                                             unsigned long long* n_runs, size_t runs_cap, uint32_t* error) {
    const size_t end = divert_run_end<U, XF>(d, n, i, shift);
    const size_t len = end - i;
    if (len <= (size_t)DIVERT_SHORT) {
        divert_sort_short<U, XF>(d, i, len);
    } else {
        const unsigned long long slot = atomicAdd(n_runs, 1ull);
        if (slot < runs_cap) runs[slot] = i;
        else atomicOr(error, ERR_BOUNDS);  // cannot happen: a listed run holds more than DIVERT_SHORT keys
    }
}

// KPT keys a lane, consecutive (16-byte loads when the keys are aligned), a
// warp 32 * KPT consecutive keys per step. A key starts a run of two or more
// when its prefix differs from the key before and equals the key after; the
// key after that tells whether the run has exactly two keys, which are then
// ordered from registers (most runs); longer runs take the slow path.
template <typename U, int XF>
__global__ void __launch_bounds__(256, 4) k_divert_runs(const Plan* __restrict__ plan, U* d, size_t n,
                                                     unsigned long long* __restrict__ runs,
                                                     unsigned long long* __restrict__ n_runs, size_t runs_cap,
                                                     uint32_t* __restrict__ error, int vec_ok) {
    dep_wait();
    dep_release();
    if (plan->mode != MODE_SORT || plan->divert_shift <= 0) return;
    constexpr int KPT = 32 / sizeof(U);  // two 16-byte vectors
    constexpr int W = 32 * KPT;          // keys a warp step
    const int shift = plan->divert_shift;
    auto pre = [&](U v) { return (unsigned long long)to_key<U, XF>(v) >> shift; };
    const int lane = threadIdx.x & 31;
    const size_t gw = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
    for (size_t wb = gw * W; wb < n; wb += nw * W) {  // warp-uniform
        const size_t i0 = wb + (size_t)lane * KPT;
        U k[KPT + 2];  // this lane's keys, then the next two
        if (vec_ok && i0 + KPT <= n) {
            const uint4* p = reinterpret_cast<const uint4*>(d + i0);
            union {
                uint4 q[2];
                U e[KPT];
            } u;
            u.q[0] = p[0];
            u.q[1] = p[1];
#pragma unroll
            for (int e = 0; e < KPT; ++e) k[e] = u.e[e];
        } else {
#pragma unroll
            for (int e = 0; e < KPT; ++e) k[e] = i0 + e < n ? d[i0 + e] : (U)0;
        }
        U prev = __shfl_up_sync(0xffffffffu, k[KPT - 1], 1);
        k[KPT] = __shfl_down_sync(0xffffffffu, k[0], 1);
        k[KPT + 1] = __shfl_down_sync(0xffffffffu, k[1], 1);
        if (lane == 0 && i0 > 0 && i0 < n) prev = d[i0 - 1];
        if (lane == 31) {
            if (i0 + KPT < n) k[KPT] = d[i0 + KPT];
            if (i0 + KPT + 1 < n) k[KPT + 1] = d[i0 + KPT + 1];
        }
        unsigned long long pp = pre(prev);
        unsigned long long p[KPT + 2];
#pragma unroll
        for (int e = 0; e < KPT + 2; ++e) p[e] = pre(k[e]);
#pragma unroll
        for (int e = 0; e < KPT; ++e) {
            const size_t i = i0 + e;
            const bool start = i == 0 || pp != p[e];
            pp = p[e];
            if (i + 1 >= n || !start || p[e + 1] != p[e]) continue;
            if (i + 2 >= n || p[e + 2] != p[e]) {
                // exactly two keys
                if (to_key<U, XF>(k[e]) > to_key<U, XF>(k[e + 1])) {
                    d[i] = k[e + 1];
                    d[i + 1] = k[e];
                }
            } else {
                divert_long_run<U, XF>(d, n, i, shift, runs, n_runs, runs_cap, error);
            }
        }
    }
}

template <typename U, int XF>
__global__ void __launch_bounds__(SEG_THREADS, 1)
    k_divert_long(const Plan* __restrict__ plan, U* d, U* __restrict__ alt, size_t n,
                  const unsigned long long* __restrict__ runs, const unsigned long long* __restrict__ n_runs,
                  unsigned int* __restrict__ counter, uint32_t* __restrict__ error) {
    dep_wait();
    dep_release();
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
