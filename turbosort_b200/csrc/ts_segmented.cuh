// ts_segmented.cuh — many independent slices sorted in one persistent launch.
//
// The crate sorts each slice with its own call (the pattern of its
// small_batches benchmark, benches/sort_bench.rs:229-250, and of
// compare/src/main.rs:49-51); here a batch of slices given by offsets is
// sorted at once. k_seg_bin puts each segment in a length bin; k_seg_sort is
// one persistent launch whose CTAs take work items largest first:
//   LARGE  one segment above the register capacity: one MSD digit pass over
//          its key range in shared memory (msd_sort, 32- and 64-bit keys)
//          while it fits there, else a CTA-level LSD over its varying digits, tile by tile
//          through a global scratch copy (the segment stays in L2), with
//          running per-digit offsets;
//   BLOCK  one segment of up to CAP keys, sorted entirely on chip: keys in
//          registers, one shared staging buffer, one stable pass per varying
//          digit (radix with 4- or 8-bit digits) or a bitonic network, as the
//          tuned configuration of its length bin says;
//   WARP   up to 32 segments of at most 32 keys, one per warp, bitonic in
//          registers with shuffles.
// Every result equals the crate's sort of that slice (src/dispatch.rs:31):
// the sorted order of radix keys is unique.
#pragma once

#include <type_traits>

#include "ts_common.cuh"
#include "ts_onesweep.cuh"
#include "ts_small.cuh"

namespace ts {

constexpr int SEG_THREADS = 1024;
constexpr int SEG_WARPS = SEG_THREADS / 32;
constexpr int SEG_BLOCK_BINS = 4;  // BLOCK length bins: (32,256] (256,1024] (1024,4096] (4096,CAP]
constexpr int SEG_BIN_WARP = SEG_BLOCK_BINS;
constexpr int SEG_BIN_LARGE = SEG_BLOCK_BINS + 1;
constexpr int SEG_NBINS = SEG_BLOCK_BINS + 2;

// The on-chip method of a BLOCK bin. SEG_MSD is the LARGE segments' routine
// (one MSD pass over the key range in shared memory, then each key to its
// place inside its sub-range);
// SEG_WARP8 (the first bin, up to 256 keys) and SEG_WARP32 (the second bin,
// up to 1024 keys of at most 4 bytes) sort 32 segments a CTA, one a warp, in
// registers (8 or 32 keys a lane; 16 when a segment has at most 512).
// SEG_MSD_GROUPS (the third and fourth bins, keys of 4 and 8 bytes) runs the
// MSD routine in thread groups, four segments a CTA in the third bin (up to
// 4096 keys) and two in the fourth.
enum SegMethod : int {
    SEG_BITONIC = 0, SEG_RADIX4 = 1, SEG_RADIX8 = 2, SEG_MSD = 3, SEG_WARP8 = 4, SEG_WARP32 = 5, SEG_MSD_GROUPS = 6
};
constexpr int SEG_METHODS = 7;
__host__ __device__ inline bool seg_method_ok(int bin, int m, int key_bytes) {
    if (m < 0 || m >= SEG_METHODS) return false;
    if (m == SEG_WARP8) return bin == 0;
    if (m == SEG_WARP32) return bin == 1 && key_bytes <= 4;
    if (m == SEG_MSD_GROUPS) return (bin == 2 || bin == 3) && key_bytes >= 4;
    return true;
}
// segments a work item of this bin and method takes
__host__ __device__ inline int seg_per_item(int bin, int m) {
    if ((bin == 0 && m == SEG_WARP8) || (bin == 1 && m == SEG_WARP32)) return SEG_WARPS;
    if (m == SEG_MSD_GROUPS) return bin == 2 ? 4 : 2;
    return 1;
}
__host__ __device__ inline bool seg_grouped(int bin, int m) { return seg_per_item(bin, m) > 1; }

template <typename U>
struct SegCfg {
    static constexpr int IPT = sizeof(U) == 8 ? 8 : 16;  // keys per thread held in registers
    static constexpr int CAP = SEG_THREADS * IPT;        // largest segment sorted on chip
    static constexpr int LARGE_IPT = sizeof(U) == 8 ? 8 : 16;
    static constexpr int LARGE_TILE = SEG_THREADS * LARGE_IPT;
};

struct SegPlan {
    unsigned int count[SEG_NBINS];  // segments per bin
    unsigned int items;             // work items in total
    int method[SEG_BLOCK_BINS];     // tuned method per BLOCK bin
    unsigned int pad[6];
};

__host__ __device__ inline int seg_bin_of(unsigned long long len, int cap) {
    if (len <= 32) return SEG_BIN_WARP;
    if (len > (unsigned long long)cap) return SEG_BIN_LARGE;
    if (len <= 256) return 0;
    if (len <= 1024) return 1;
    if (len <= 4096) return 2;
    return 3;
}

// Work items, largest first: LARGE segments, BLOCK bins from the longest
// down (the first BLOCK bin in groups of SEG_WARPS segments when it takes
// SEG_WARP8), then groups of SEG_WARPS tiny segments.
__device__ __forceinline__ void seg_item(const SegPlan& p, unsigned int item, int* bin, unsigned int* first) {
    unsigned int base = 0;
    if (item < base + p.count[SEG_BIN_LARGE]) {
        *bin = SEG_BIN_LARGE;
        *first = item - base;
        return;
    }
    base += p.count[SEG_BIN_LARGE];
    for (int b = SEG_BLOCK_BINS - 1; b >= 0; --b) {
        const unsigned int per = (unsigned int)seg_per_item(b, p.method[b]);
        const unsigned int items = (p.count[b] + per - 1) / per;
        if (item < base + items) {
            *bin = b;
            *first = (item - base) * per;
            return;
        }
        base += items;
    }
    *bin = SEG_BIN_WARP;
    *first = (item - base) * SEG_WARPS;
}

struct SegMethods {
    int m[SEG_BLOCK_BINS];
};

static __global__ void k_seg_items(SegPlan* plan, SegMethods methods) {
    if (threadIdx.x == 0) {
        unsigned int t = plan->count[SEG_BIN_LARGE] + (plan->count[SEG_BIN_WARP] + SEG_WARPS - 1) / SEG_WARPS;
        for (int b = 0; b < SEG_BLOCK_BINS; ++b) {
            plan->method[b] = methods.m[b];
            const unsigned int per = (unsigned int)seg_per_item(b, methods.m[b]);
            t += (plan->count[b] + per - 1) / per;
        }
        plan->items = t;
    }
}

// ---- WARP: bitonic network over 32 lanes ---------------------------------
template <typename U, int XF>
__device__ __forceinline__ void seg_warp_sort(const U* in, U* seg, int len, int lane) {
    U v = lane < len ? to_key<U, XF>(in[lane]) : (U)~(U)0;
#pragma unroll
    for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            const U o = __shfl_xor_sync(0xffffffffu, v, j);
            const bool keep_min = ((lane & j) == 0) == ((lane & k) == 0);
            v = keep_min ? (o < v ? o : v) : (o > v ? o : v);
        }
    }
    if (lane < len) seg[lane] = from_key<U, XF>(v);
}

// ---- BLOCK: on-chip sorts ---------------------------------------------------
// Bitonic over the next power of two in shared memory.
template <typename U, int XF>
__device__ void seg_block_bitonic(const U* in, U* seg, int len, U* sm) {
    int p2 = 1;
    while (p2 < len) p2 <<= 1;
    for (int i = threadIdx.x; i < p2; i += SEG_THREADS) sm[i] = i < len ? to_key<U, XF>(in[i]) : (U)~(U)0;
    __syncthreads();
    for (int k = 2; k <= p2; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < p2 / 2; i += SEG_THREADS) {
                // the i-th compare-exchange pair of this step
                const int lo = ((i & ~(j - 1)) << 1) | (i & (j - 1));
                const int hi = lo | j;
                const bool up = (lo & k) == 0;
                const U a = sm[lo], b = sm[hi];
                if ((a > b) == up) {
                    sm[lo] = b;
                    sm[hi] = a;
                }
            }
            __syncthreads();
        }
    }
    for (int i = threadIdx.x; i < len; i += SEG_THREADS) seg[i] = from_key<U, XF>(sm[i]);
}

// One stable pass of the on-chip LSD: keys in registers (warp-striped: item i
// of lane l of warp w is key w*32*IPT + i*32 + l), written to their sorted
// places in `sm`. cnt is [SEG_WARPS][RADIX].
template <typename U, int BITS, int IPT>
__device__ __forceinline__ void seg_rank_pass(const U (&k)[IPT], int wbase, int ipt, int len, int shift, U* sm,
                                              uint32_t* cnt, int* warp_tot, const PeerMasks<BITS>& pm,
                                              uint32_t* lstart_out = nullptr, uint32_t* count_out = nullptr) {
    constexpr int RADIX = 1 << BITS;
    constexpr uint32_t MASK = RADIX - 1;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    uint32_t* my_cnt = cnt + warp * RADIX;
    for (int i = tid; i < SEG_WARPS * RADIX; i += SEG_THREADS) cnt[i] = 0;
    __syncthreads();
#pragma unroll
    for (int i = 0; i < IPT; ++i)
        if (i < ipt && wbase + i * 32 < len) atomicAdd(&my_cnt[digit_of(k[i], shift, MASK)], 1u);
    __syncthreads();
    // per digit: prefix over warps; then an exclusive scan over digits
    uint32_t own = 0;
    for (int r = tid; r < RADIX; r += SEG_THREADS) {
        uint32_t s = 0;
        for (int w = 0; w < SEG_WARPS; ++w) {
            const uint32_t c = cnt[w * RADIX + r];
            cnt[w * RADIX + r] = s;
            s += c;
        }
        own = s;  // RADIX <= SEG_THREADS: one digit per thread
    }
    uint32_t x = own;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[warp] = (int)x;
    __syncthreads();
    if (tid < RADIX) {
        uint32_t run = x - own;
        for (int w = 0; w < warp; ++w) run += (uint32_t)warp_tot[w];
        for (int w = 0; w < SEG_WARPS; ++w) cnt[w * RADIX + tid] += run;
        if (lstart_out) {
            lstart_out[tid] = run;
            count_out[tid] = own;
        }
    }
    __syncthreads();
    const uint32_t lt = lanemask_lt();
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
        if (i >= ipt) break;  // uniform: ipt is the same for the whole block
        const bool valid = wbase + i * 32 < len;
        const uint32_t d = digit_of(k[i], shift, MASK);
        const uint32_t peers = pm.peers(d) & __ballot_sync(0xffffffffu, valid);
        if (valid) {
            const uint32_t c = my_cnt[d];
            my_cnt[d] = c + __popc(peers);
            sm[c + __popc(peers & lt)] = k[i];
        }
        __syncwarp();
    }
    __syncthreads();
}

template <typename U, int XF, int BITS>
__device__ void seg_block_radix(const U* in, U* seg, int len, U* sm, uint32_t* cnt, int* warp_tot,
                                unsigned long long* red) {
    constexpr int IPT = SegCfg<U>::IPT;
    constexpr int ND = (Bits<U>::W + BITS - 1) / BITS;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // spread the keys over the warps: each warp takes a contiguous run
    const int ipt = (len + SEG_THREADS - 1) / SEG_THREADS;  // items per lane actually used
    const int wbase = warp * 32 * ipt + lane;
    PeerMasks<BITS> pm;
    pm.init(lane);
    U k[IPT];
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
        const int idx = wbase + i * 32;
        k[i] = (i < ipt && idx < len) ? to_key<U, XF>(in[idx]) : (U)0;
    }
    if (threadIdx.x == 0) *red = 0;
    __syncthreads();
    // the bits in which some key differs from the first: only those digits get a pass
    const U first = to_key<U, XF>(in[0]);
    unsigned long long d = 0;
#pragma unroll
    for (int i = 0; i < IPT; ++i)
        if (i < ipt && wbase + i * 32 < len) d |= (unsigned long long)(k[i] ^ first);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) d |= __shfl_xor_sync(0xffffffffu, d, o);
    if (lane == 0) atomicOr(red, d);
    __syncthreads();
    const unsigned long long vary = *red;
    for (int p = 0; p < ND; ++p) {
        if (((vary >> (p * BITS)) & ((1ull << BITS) - 1)) == 0) continue;
        seg_rank_pass<U, BITS, IPT>(k, wbase, ipt, len, p * BITS, sm, cnt, warp_tot, pm);
        // reload in the same warp-striped layout for the next pass
#pragma unroll
        for (int i = 0; i < IPT; ++i) {
            const int idx = wbase + i * 32;
            k[i] = (i < ipt && idx < len) ? sm[idx] : (U)0;
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
        const int idx = wbase + i * 32;
        if (i < ipt && idx < len) seg[idx] = from_key<U, XF>(k[i]);
    }
}

// ---- LARGE: a CTA-level LSD through the segment's scratch copy ------------
struct SegSmem {
    // offsets of the shared-memory areas (bytes) for key type U
    template <typename U>
    static constexpr size_t sm_bytes() { return (size_t)SegCfg<U>::CAP * sizeof(U); }
    template <typename U>
    static constexpr size_t cnt_off() { return sm_bytes<U>(); }
    template <typename U>
    static constexpr size_t hist_off() { return cnt_off<U>() + (size_t)SEG_WARPS * 256 * 4; }
    template <typename U>
    static constexpr size_t run_off() { return hist_off<U>() + (size_t)8 * 256 * 4; }
    template <typename U>
    static constexpr size_t misc_off() { return run_off<U>() + (size_t)3 * 256 * 4; }
    template <typename U>
    static constexpr size_t bytes() { return misc_off<U>() + 512; }
};

template <typename U, int XF>
__device__ void seg_large_sort(const U* in, U* seg, U* alt, int len, U* sm, uint32_t* cnt, int* warp_tot,
                               unsigned long long* red, uint32_t* hist, uint32_t* run, uint32_t* lst, uint32_t* tcnt) {
    constexpr int RADIX = 256;
    constexpr int ND = (int)sizeof(U);
    constexpr int IPT = SegCfg<U>::LARGE_IPT;
    constexpr int TILE = SegCfg<U>::LARGE_TILE;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    PeerMasks<8> pm;
    pm.init(lane);
    // 1. one read: the bits that vary and the histogram of every digit
    for (int i = tid; i < ND * RADIX; i += SEG_THREADS) hist[i] = 0;
    if (tid == 0) *red = 0;
    __syncthreads();
    const U first = to_key<U, XF>(in[0]);
    unsigned long long d = 0;
    for (int i = tid; i < len; i += SEG_THREADS) {
        const U k = to_key<U, XF>(in[i]);
        d |= (unsigned long long)(k ^ first);
#pragma unroll
        for (int p = 0; p < ND; ++p) atomicAdd(&hist[p * RADIX + digit_of(k, p * 8, RADIX - 1)], 1u);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) d |= __shfl_xor_sync(0xffffffffu, d, o);
    if (lane == 0) atomicOr(red, d);
    __syncthreads();
    const unsigned long long vary = *red;
    int last_p = -1;
    for (int p = 0; p < ND; ++p)
        if ((vary >> (p * 8)) & 0xff) last_p = p;
    // 2. one pass per varying digit, tile by tile, with running digit offsets
    bool in_alt = false, first_pass = true;
    for (int p = 0; p < ND; ++p) {
        if (((vary >> (p * 8)) & 0xff) == 0) continue;
        const U* src = first_pass ? in : (in_alt ? alt : seg);
        U* dst = in_alt ? seg : alt;
        const bool last = p == last_p;
        // exclusive scan of this digit's histogram into run[]
        {
            const uint32_t own = tid < RADIX ? hist[p * RADIX + tid] : 0u;
            uint32_t x = own;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            if (lane == 31) warp_tot[warp] = (int)x;
            __syncthreads();
            if (tid < RADIX) {
                uint32_t r = x - own;
                for (int w = 0; w < warp; ++w) r += (uint32_t)warp_tot[w];
                run[tid] = r;
            }
            __syncthreads();
        }
        for (int t0 = 0; t0 < len; t0 += TILE) {
            const int tn = min(TILE, len - t0);
            const int ipt = (tn + SEG_THREADS - 1) / SEG_THREADS;
            const int wbase = warp * 32 * ipt + lane;
            U k[IPT];
#pragma unroll
            for (int i = 0; i < IPT; ++i) {
                const int idx = wbase + i * 32;
                U v = (i < ipt && idx < tn) ? src[t0 + idx] : (U)0;
                k[i] = first_pass ? to_key<U, XF>(v) : v;
            }
            seg_rank_pass<U, 8, IPT>(k, wbase, ipt, tn, p * 8, sm, cnt, warp_tot, pm, lst, tcnt);
            for (int s2 = tid; s2 < tn; s2 += SEG_THREADS) {
                const U key = sm[s2];
                const uint32_t dg = digit_of(key, p * 8, RADIX - 1);
                dst[run[dg] + (uint32_t)s2 - lst[dg]] = last ? from_key<U, XF>(key) : key;
            }
            __syncthreads();
            if (tid < RADIX) run[tid] += tcnt[tid];
            __syncthreads();
        }
        in_alt = !in_alt;
        first_pass = false;
    }
    if (in_alt) {
        for (int i = tid; i < len; i += SEG_THREADS) seg[i] = alt[i];
    } else if (first_pass && in != seg) {  // every key equal: nothing moved yet
        for (int i = tid; i < len; i += SEG_THREADS) seg[i] = in[i];
    }
}

// ---- MSD: one digit pass over a segment's key range, in shared memory -------
// A segment of up to MsdSmem<U>::cap keys (24.8K of 8 bytes, 49.6K of 4) is
// sorted with one MSD digit pass: its keys' range [kmin, kmax] is cut into up
// to 2^14 equal sub-ranges (a monotone map, so the sub-ranges are ordered;
// about one key each), keys are counted and placed by sub-range in shared
// memory with 16-bit counters, and each key goes to its sorted place inside
// its sub-range (msd_finish).
// Longer segments, or segments whose keys crowd one sub-range (MSD_SUB_MAX
// keys), take the CTA-level LSD through `scratch`. src may equal dst.
constexpr int MSD_SMEM = 227 * 1024;
constexpr int MSD_SUB_BITS = 14;
constexpr int MSD_SUB_MAX = 128;

// fn(i, src[i]) for this thread's share of 0..len-1, its loads issued a
// group at a time (one segment is read by one CTA: latency, not bandwidth,
// bounds a plain loop)
template <typename U, typename Fn>
__device__ __forceinline__ void msd_for_keys(const U* __restrict__ src, int len, Fn fn) {
    constexpr int G = 32 / sizeof(U);
    for (int base = threadIdx.x; base < len; base += 1024 * G) {
        U v[G];
#pragma unroll
        for (int e = 0; e < G; ++e) {
            const int i = base + e * 1024;
            v[e] = i < len ? src[i] : (U)0;
        }
#pragma unroll
        for (int e = 0; e < G; ++e) {
            const int i = base + e * 1024;
            if (i < len) fn(i, v[e]);
        }
    }
}

// The run of sub-ranges d0 .. d0 + per - 1 of a placement whose packed
// 16-bit counters (wd) now hold each sub-range's end, insertion-sorted as
// one run: keys are in order from one sub-range to the next, so only keys
// inside a sub-range (about one or two) move. (Sorting each sub-range on its
// own, two or three keys from registers, measured slower: 2.90 against 2.50
// ms for 10,485 segments of 30,000 keys.)
template <typename U>
__device__ __forceinline__ void msd_insert_run(U* sk, const unsigned int* wd, int d0, int per) {
    auto end_of = [&](int d) { return (int)((wd[d >> 1] >> ((d & 1) * 16)) & 0xffffu); };
    const int r0 = d0 == 0 ? 0 : end_of(d0 - 1);
    const int r1 = end_of(d0 + per - 1);
    for (int i = r0 + 1; i < r1; ++i) {
        const U v = sk[i];
        int j = i - 1;
        while (j >= r0 && sk[j] > v) {
            sk[j + 1] = sk[j];
            --j;
        }
        sk[j + 1] = v;
    }
}

// The keys of a placement (grouped by sub-range, in any order inside a
// sub-range; the packed 16-bit counters wd hold each sub-range's end), each
// written to its sorted place in dst: its sub-range's start plus the number
// of the sub-range's keys below it, or equal to it and placed before it.
// Thread `tid` of `nthreads` takes positions tid, tid + nthreads, ...: the
// lanes of a warp hold neighbouring positions, so the sub-ranges they scan
// are neighbours (their shared reads fall in different banks) and their
// stores land in one short span of dst. Used for 8-byte keys, whose
// insertion runs (above) start about a run length apart, so that a warp's
// reads of two-word keys meet in few banks; for 4-byte keys, with up to
// three keys a sub-range, the runs measured faster (see msd_finish).
template <typename U, int XF, typename Digit>
__device__ __forceinline__ void msd_emit(const U* sk, const unsigned int* wd, int len, int tid, int nthreads,
                                         Digit digit, U* __restrict__ dst) {
    auto end_of = [&](int d) { return (int)((wd[d >> 1] >> ((d & 1) * 16)) & 0xffffu); };
    for (int p = tid; p < len; p += nthreads) {
        const U v = sk[p];
        const int d = digit((unsigned long long)v);
        const int s = d == 0 ? 0 : end_of(d - 1);
        const int e = end_of(d);
        int r = 0;
        if (e - s > 1) {
            for (int q = s; q < e; ++q) {
                const U u = sk[q];
                r += (u < v || (u == v && q < p)) ? 1 : 0;
            }
        }
        dst[s + r] = from_key<U, XF>(v);
    }
}

// The last step of the MSD routine, once the keys are placed by sub-range:
// every key to its sorted place in dst. Measured on a B200: 8-byte keys by
// rank (msd_emit; the learned finish of 2^28 keys in 16,384 buckets gained
// about 0.1 ms), keys of up to 4 bytes by insertion over each thread's run of
// sub-ranges and a copy (100,000 segments of 4-byte keys: 6.38 ms by rank
// against 5.83 ms this way). `owners` threads own `per` sub-ranges each;
// `sync` is the caller's barrier, taken between the insertion runs and the
// copy, and the caller synchronises again after the call.
template <typename U, int XF, typename Digit, typename Sync>
__device__ __forceinline__ void msd_finish(U* sk, const unsigned int* wd, int len, int tid, int nthreads, int owners,
                                           int per, Digit digit, U* __restrict__ dst, Sync sync) {
    if constexpr (sizeof(U) == 8) {
        msd_emit<U, XF>(sk, wd, len, tid, nthreads, digit, dst);
    } else {
        if (tid < owners) msd_insert_run<U>(sk, wd, tid * per, per);
        sync();
        for (int i = tid; i < len; i += nthreads) dst[i] = from_key<U, XF>(sk[i]);
    }
}

template <typename U>
struct MsdSmem {
    static constexpr size_t misc = MSD_SMEM - 1024;                        // warp totals, reductions, item ids
    static constexpr size_t words = misc - (size_t)(1 << MSD_SUB_BITS) * 2;  // 16-bit counters, two a word
    static constexpr int cap = (int)(words / sizeof(U)) < 65535 ? (int)(words / sizeof(U)) : 65535;
};

// One segment, by the whole CTA (1024 threads); `sm` is MSD_SMEM bytes of
// shared memory; `scratch` has room for len keys, or is null when src may be
// overwritten (it then serves as the CTA LSD's second buffer).
template <typename U, int XF>
__device__ void msd_core(const U* src, U* dst, U* scratch, int len, unsigned char* sm) {
    using M = MsdSmem<U>;
    U* sk = reinterpret_cast<U*>(sm);
    unsigned int* wd = reinterpret_cast<unsigned int*>(sm + M::words);  // counter d: half (d & 1) of wd[d >> 1]
    int* misc = reinterpret_cast<int*>(sm + M::misc);
    int* warp_tot = misc;                                                         // [32]
    unsigned long long* red = reinterpret_cast<unsigned long long*>(misc + 32);  // [4]
    // the CTA-level LSD's areas, inside the key area (unused while it runs)
    uint32_t* l_cnt = reinterpret_cast<uint32_t*>(sm + (size_t)SegCfg<U>::LARGE_TILE * sizeof(U));
    uint32_t* l_hist = l_cnt + SEG_WARPS * 256;
    uint32_t* l_run = l_hist + 8 * 256;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    auto half = [](unsigned int w, int d) { return (w >> ((d & 1) * 16)) & 0xffffu; };
    if (len <= 1) {
        if (len == 1 && tid == 0) dst[0] = src[0];
        return;
    }
    if (tid == 0) red[2] = 0ull;
    bool large = len > M::cap;
    unsigned long long kmin = 0, kmax = 0;
    int bits = 1;
    if (!large) {
        // pass 1: the bucket's key range, and a copy of its keys in the
        // placement area (read by pass 2 instead of a second read from L2)
        if (tid == 0) {
            red[0] = ~0ull;
            red[1] = 0ull;
        }
        __syncthreads();
        unsigned long long mn = ~0ull, mx = 0ull;
        msd_for_keys<U>(src, len, [&](int i, U v) {
            const U k = to_key<U, XF>(v);
            sk[i] = k;
            mn = (unsigned long long)k < mn ? (unsigned long long)k : mn;
            mx = (unsigned long long)k > mx ? (unsigned long long)k : mx;
        });
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long x = __shfl_xor_sync(0xffffffffu, mn, o);
            const unsigned long long y = __shfl_xor_sync(0xffffffffu, mx, o);
            mn = x < mn ? x : mn;
            mx = y > mx ? y : mx;
        }
        if (lane == 0) {
            atomicMin(&red[0], mn);
            atomicMax(&red[1], mx);
        }
        __syncthreads();
        kmin = red[0];
        kmax = red[1];
        if (kmin == kmax) {  // every key equal
            msd_for_keys<U>(src, len, [&](int i, U v) { dst[i] = v; });
            __syncthreads();
            return;
        }
        while (bits < MSD_SUB_BITS && (2 << bits) <= len) ++bits;  // about one or two keys a sub-range
    }
    const int nb = 1 << bits;
    const int per = nb >= 2048 ? nb / 1024 : 2;  // counters a thread scans and sorts (even)
    const int owners = nb / per;
    const float scale = large ? 0.f : (float)nb / __ull2float_ru(kmax - kmin);
    auto digit = [&](unsigned long long k) { return min(nb - 1, (int)(__ull2float_rz(k - kmin) * scale)); };
    if (!large) {
        // pass 2: counts per sub-range
        for (int w = tid; w < nb / 2; w += 1024) wd[w] = 0u;
        __syncthreads();
        for (int i = tid; i < len; i += 1024) {
            const int d = digit((unsigned long long)sk[i]);
            atomicAdd(&wd[d >> 1], 1u << ((d & 1) * 16));
        }
        __syncthreads();
        // exclusive scan of the counters (each owner a run of `per`), their largest
        unsigned int sum = 0, m = 0;
        if (tid < owners)
            for (int q = 0; q < per / 2; ++q) {
                const unsigned int w = wd[tid * (per / 2) + q];
                sum += (w & 0xffffu) + (w >> 16);
                m = max(m, max(w & 0xffffu, w >> 16));
            }
        unsigned int x = sum;
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (lane == 31) warp_tot[warp] = (int)x;
        if (lane == 0) atomicMax(reinterpret_cast<unsigned int*>(&red[2]), m);
        __syncthreads();
        unsigned int run = x - sum;
        for (int w = 0; w < warp; ++w) run += (unsigned int)warp_tot[w];
        if (tid < owners)
            for (int q = 0; q < per / 2; ++q) {
                const unsigned int w = wd[tid * (per / 2) + q];
                const unsigned int s0 = run, s1 = run + (w & 0xffffu);
                run = s1 + (w >> 16);
                wd[tid * (per / 2) + q] = s0 | (s1 << 16);  // starts, which become cursors
            }
        __syncthreads();
        large = reinterpret_cast<unsigned int*>(&red[2])[0] > (unsigned int)MSD_SUB_MAX;
        __syncthreads();
        if (tid == 0) red[2] = 0ull;
    }
    if (large) {
        if (scratch == nullptr) {
            // src is expendable (msd_split's parts): sort in dst, with src as
            // the LSD's second buffer
            for (int i = tid; i < len; i += 1024) dst[i] = src[i];
            __syncthreads();
            seg_large_sort<U, XF>(dst, dst, const_cast<U*>(src), len, sk, l_cnt, warp_tot, &red[3], l_hist, l_run,
                                  l_run + 256, l_run + 512);
        } else {
            seg_large_sort<U, XF>(src, dst, scratch, len, sk, l_cnt, warp_tot, &red[3], l_hist, l_run, l_run + 256,
                                  l_run + 512);
        }
        __syncthreads();
        return;
    }
    // pass 3: place keys by sub-range; each counter ends at its sub-range's end
    msd_for_keys<U>(src, len, [&](int, U v) {
        const U k = to_key<U, XF>(v);
        const int d = digit((unsigned long long)k);
        sk[half(atomicAdd(&wd[d >> 1], 1u << ((d & 1) * 16)), d)] = k;
    });
    __syncthreads();
    // pass 4: every key to its sorted place (out of order only inside
    // sub-ranges, of about one or two keys)
    msd_finish<U, XF>(sk, wd, len, tid, 1024, owners, per, digit, dst, [] { __syncthreads(); });
    __syncthreads();
}

// Segments of up to MSD_SPLIT_PARTS times the on-chip capacity: one coarse
// MSD pass cuts the key range into MSD_COARSE equal sub-ranges; with T the
// capacity less the fullest sub-range, sub-range r goes to part start_r / T
// (start_r: keys in the sub-ranges before it), so every part holds at most
// the capacity unless one narrow key range alone holds more; the keys go to
// their part in `scratch` (each warp groups its keys by part, so a part's keys
// from one warp land at consecutive addresses), and each part is sorted from
// there into its place in dst: by msd_core, whose CTA-level LSD takes a part
// too crowded for the sub-range pass. The parts are in key order, so the
// segment ends up sorted.
constexpr int MSD_SPLIT_PARTS = 4;
constexpr int MSD_COARSE = 4096;
constexpr int MSD_MAX_PARTS = 16;  // ceil(len / T) with T >= len / 16

template <typename U, int XF>
__device__ void msd_split(const U* src, U* dst, U* scratch, int len, unsigned char* sm) {
    using M = MsdSmem<U>;
    uint32_t* cur = reinterpret_cast<uint32_t*>(sm);                       // [MSD_COARSE] counts, then starts
    unsigned char* part_of = sm + MSD_COARSE * 4;                          // [MSD_COARSE]
    int* misc = reinterpret_cast<int*>(sm + M::misc);
    int* warp_tot = misc;                                                  // [32]
    unsigned long long* red = reinterpret_cast<unsigned long long*>(misc + 32);  // [4]
    int* bounds = misc + 64;                                               // [MSD_MAX_PARTS + 1]
    int* pcur = misc + 64 + MSD_MAX_PARTS + 1;                             // [MSD_MAX_PARTS]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // the key range
    if (tid == 0) {
        red[0] = ~0ull;
        red[1] = 0ull;
        red[2] = 0ull;
    }
    for (int i = tid; i < MSD_COARSE; i += 1024) cur[i] = 0u;
    __syncthreads();
    unsigned long long mn = ~0ull, mx = 0ull;
    msd_for_keys<U>(src, len, [&](int, U v) {
        const unsigned long long k = (unsigned long long)to_key<U, XF>(v);
        mn = k < mn ? k : mn;
        mx = k > mx ? k : mx;
    });
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long x = __shfl_xor_sync(0xffffffffu, mn, o);
        const unsigned long long y = __shfl_xor_sync(0xffffffffu, mx, o);
        mn = x < mn ? x : mn;
        mx = y > mx ? y : mx;
    }
    if (lane == 0) {
        atomicMin(&red[0], mn);
        atomicMax(&red[1], mx);
    }
    __syncthreads();
    const unsigned long long kmin = red[0], kmax = red[1];
    if (kmin == kmax) {  // every key equal
        msd_for_keys<U>(src, len, [&](int i, U v) { dst[i] = v; });
        __syncthreads();
        return;
    }
    const float scale = (float)MSD_COARSE / __ull2float_ru(kmax - kmin);
    auto coarse = [&](U v) {
        return min(MSD_COARSE - 1, (int)(__ull2float_rz((unsigned long long)to_key<U, XF>(v) - kmin) * scale));
    };
    msd_for_keys<U>(src, len, [&](int, U v) { atomicAdd(&cur[coarse(v)], 1u); });
    __syncthreads();
    // exclusive scan (four sub-ranges a thread) and the fullest sub-range
    uint32_t c4[4], sum = 0, mc = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        c4[q] = cur[tid * 4 + q];
        sum += c4[q];
        mc = max(mc, c4[q]);
    }
    uint32_t x = sum;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    for (int o = 16; o > 0; o >>= 1) mc = max(mc, __shfl_xor_sync(0xffffffffu, mc, o));
    if (lane == 31) warp_tot[warp] = (int)x;
    if (lane == 0) atomicMax(reinterpret_cast<unsigned int*>(&red[2]), mc);
    if (tid <= MSD_MAX_PARTS) bounds[tid] = len;
    __syncthreads();
    uint32_t run = x - sum;
    for (int w = 0; w < warp; ++w) run += (uint32_t)warp_tot[w];
    const int maxc = (int)reinterpret_cast<unsigned int*>(&red[2])[0];
    const int target = max(M::cap - maxc, (len + MSD_MAX_PARTS - 1) / MSD_MAX_PARTS);
    // sub-range r's part, and each part's first key (a part that receives
    // no sub-range starts where the next one does)
    int prev_part = -1;
    if (tid > 0)  // the part of the previous thread's last sub-range
        prev_part = min(MSD_MAX_PARTS - 1, (int)((run - cur[tid * 4 - 1]) / (uint32_t)target));
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int p = min(MSD_MAX_PARTS - 1, (int)(run / (uint32_t)target));
        part_of[tid * 4 + q] = (unsigned char)p;
        if (p != prev_part) atomicMin(&bounds[p], (int)run);
        prev_part = p;
        run += c4[q];
    }
    __syncthreads();
    if (tid == 0) {
        for (int p = MSD_MAX_PARTS - 1; p >= 0; --p) bounds[p] = min(bounds[p], bounds[p + 1]);
        bounds[0] = 0;
        for (int p = 0; p < MSD_MAX_PARTS; ++p) pcur[p] = bounds[p];
    }
    __syncthreads();
    // place the keys by part: a warp's keys of one part at consecutive places
    PeerMasks<4> pm;
    pm.init(lane);
    const uint32_t lt = lanemask_lt();
    for (int base = warp * 32; base < len; base += 1024) {  // warp-uniform
        const int i = base + lane;
        const bool valid = i < len;
        const U v = valid ? src[i] : (U)0;
        const uint32_t p = valid ? part_of[coarse(v)] : 0u;
        const uint32_t peers = pm.peers(p) & __ballot_sync(0xffffffffu, valid);
        const int leader = __ffs(peers) - 1;
        uint32_t at = 0;
        if (valid && lane == leader) at = (uint32_t)atomicAdd(&pcur[p], __popc(peers));
        at = __shfl_sync(0xffffffffu, at, leader & 31);
        if (valid) scratch[at + __popc(peers & lt)] = v;
    }
    __syncthreads();
    for (int p = 0; p < MSD_MAX_PARTS; ++p) {
        const int a = bounds[p], b = bounds[p + 1];
        __syncthreads();  // every thread has the bounds before the part reuses shared memory
        if (b > a) msd_core<U, XF>(scratch + a, dst + a, nullptr, b - a, sm);
        __syncthreads();
    }
}

// One segment, by the whole CTA (1024 threads); `sm` is MSD_SMEM bytes of
// shared memory; `scratch` has room for len keys and is not src or dst
// (src may equal dst).
template <typename U, int XF>
__device__ void msd_sort(const U* src, U* dst, U* scratch, int len, unsigned char* sm) {
    if (len > MsdSmem<U>::cap && len <= MSD_SPLIT_PARTS * MsdSmem<U>::cap)
        msd_split<U, XF>(src, dst, scratch, len, sm);
    else msd_core<U, XF>(src, dst, scratch, len, sm);
}

// ---- several segments a CTA: the MSD routine by thread groups ---------------
// A group of G threads (its own slice of shared memory and its own named
// barrier) sorts one segment of up to SegGroup::cap keys as msd_core does:
// the key range, counts per sub-range (about one key each), placement by
// sub-range, each key to its place inside its sub-range (msd_finish). A segment
// whose keys crowd one sub-range is sorted by a bitonic network in the
// group's slice instead. The CTA runs SEG_THREADS / G groups side by side.
template <typename U, int G>
struct SegGroup {
    static constexpr int GROUPS = SEG_THREADS / G;
    static constexpr size_t slice = (size_t)MSD_SMEM / GROUPS / 128 * 128;
    static constexpr int cap = G == 256 ? 4096 : SegCfg<U>::CAP;    // the bin it serves
    static constexpr int sub_bits = G == 256 ? 12 : 14;
    static constexpr size_t key_bytes = (size_t)cap * sizeof(U);
    static constexpr size_t cnt_off = key_bytes;                     // 16-bit counters, two a word
    static constexpr size_t misc_off = cnt_off + (size_t)(1 << sub_bits) * 2;
    static_assert(misc_off + 256 <= slice, "a group's keys, counters and scratch fit its slice");
};

template <typename U, int XF, int G>
__device__ void msd_group(const U* src, U* dst, int len, unsigned char* sm, int bar) {
    using S = SegGroup<U, G>;
    U* sk = reinterpret_cast<U*>(sm);
    unsigned int* wd = reinterpret_cast<unsigned int*>(sm + S::cnt_off);
    int* warp_tot = reinterpret_cast<int*>(sm + S::misc_off);                       // [G / 32]
    unsigned long long* red = reinterpret_cast<unsigned long long*>(sm + S::misc_off + 128);  // [3]
    const int tid = threadIdx.x % G, lane = tid & 31, warp = tid >> 5;
    auto gsync = [&]() { asm volatile("bar.sync %0, %1;" ::"r"(bar), "r"(G) : "memory"); };
    auto half = [](unsigned int w, int d) { return (w >> ((d & 1) * 16)) & 0xffffu; };
    if (len <= 1) {
        if (len == 1 && tid == 0) dst[0] = src[0];
        return;
    }
    // the key range (the placement reads the segment again, from L2)
    if (tid == 0) {
        red[0] = ~0ull;
        red[1] = 0ull;
        red[2] = 0ull;
    }
    gsync();
    unsigned long long mn = ~0ull, mx = 0ull;
    for (int i = tid; i < len; i += G) {  // with a copy in the placement area, for the counts
        const U k = to_key<U, XF>(src[i]);
        sk[i] = k;
        mn = (unsigned long long)k < mn ? (unsigned long long)k : mn;
        mx = (unsigned long long)k > mx ? (unsigned long long)k : mx;
    }
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long x = __shfl_xor_sync(0xffffffffu, mn, o);
        const unsigned long long y = __shfl_xor_sync(0xffffffffu, mx, o);
        mn = x < mn ? x : mn;
        mx = y > mx ? y : mx;
    }
    if (lane == 0) {
        atomicMin(&red[0], mn);
        atomicMax(&red[1], mx);
    }
    gsync();
    const unsigned long long kmin = red[0], kmax = red[1];
    if (kmin == kmax) {  // every key equal
        for (int i = tid; i < len; i += G) dst[i] = src[i];
        gsync();
        return;
    }
    int bits = 1;
    while (bits < S::sub_bits && (2 << bits) <= len) ++bits;
    const int nb = 1 << bits;
    const int per = nb >= 2 * G ? nb / G : 2;
    const int owners = nb / per;
    const float scale = (float)nb / __ull2float_ru(kmax - kmin);
    auto digit = [&](unsigned long long k) { return min(nb - 1, (int)(__ull2float_rz(k - kmin) * scale)); };
    for (int w = tid; w < nb / 2; w += G) wd[w] = 0u;
    gsync();
    for (int i = tid; i < len; i += G) {
        const int d = digit((unsigned long long)sk[i]);
        atomicAdd(&wd[d >> 1], 1u << ((d & 1) * 16));
    }
    gsync();
    unsigned int sum = 0, m = 0;
    if (tid < owners)
        for (int q = 0; q < per / 2; ++q) {
            const unsigned int w = wd[tid * (per / 2) + q];
            sum += (w & 0xffffu) + (w >> 16);
            m = max(m, max(w & 0xffffu, w >> 16));
        }
    unsigned int x = sum;
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 31) warp_tot[warp] = (int)x;
    if (lane == 0) atomicMax(reinterpret_cast<unsigned int*>(&red[2]), m);
    gsync();
    unsigned int run = x - sum;
    for (int w = 0; w < warp; ++w) run += (unsigned int)warp_tot[w];
    if (tid < owners)
        for (int q = 0; q < per / 2; ++q) {
            const unsigned int w = wd[tid * (per / 2) + q];
            const unsigned int s0 = run, s1 = run + (w & 0xffffu);
            run = s1 + (w >> 16);
            wd[tid * (per / 2) + q] = s0 | (s1 << 16);
        }
    gsync();
    if (reinterpret_cast<unsigned int*>(&red[2])[0] > (unsigned int)MSD_SUB_MAX) {
        // crowded: a bitonic network over the slice's keys
        int p2 = 1;
        while (p2 < len) p2 <<= 1;
        for (int i = tid; i < p2; i += G) sk[i] = i < len ? to_key<U, XF>(src[i]) : (U)~(U)0;
        gsync();
        for (int k = 2; k <= p2; k <<= 1) {
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int i = tid; i < p2 / 2; i += G) {
                    const int lo = ((i & ~(j - 1)) << 1) | (i & (j - 1));
                    const int hi = lo | j;
                    const bool up = (lo & k) == 0;
                    const U a = sk[lo], b = sk[hi];
                    if ((a > b) == up) {
                        sk[lo] = b;
                        sk[hi] = a;
                    }
                }
                gsync();
            }
        }
        for (int i = tid; i < len; i += G) dst[i] = from_key<U, XF>(sk[i]);
        gsync();
        return;
    }
    // place by sub-range; each counter ends at its sub-range's end
    for (int i = tid; i < len; i += G) {
        const U k = to_key<U, XF>(src[i]);
        const int d = digit((unsigned long long)k);
        sk[half(atomicAdd(&wd[d >> 1], 1u << ((d & 1) * 16)), d)] = k;
    }
    gsync();
    // every key to its sorted place inside its sub-range
    msd_finish<U, XF>(sk, wd, len, tid, G, owners, per, digit, dst, gsync);
    gsync();
}

// One slice of up to 4096 keys of 4 or 8 bytes by one CTA: the plain sort's
// short-slice tier above the warp networks (src/small.rs:11 sorts up to 512
// with its networks; here the one-pass MSD routine takes 1025..4096 keys, a
// few barriers instead of the bitonic network's 78 stages).
template <typename U, int XF>
__global__ void __launch_bounds__(SEG_THREADS, 1) k_msd_slice(U* d, U* __restrict__ scratch, int n) {
    extern __shared__ __align__(128) unsigned char smem[];
    msd_sort<U, XF>(d, d, scratch, n, smem);
}

// ---- the persistent launch ---------------------------------------------------

template <typename U, int XF>
__global__ void __launch_bounds__(SEG_THREADS, 1)
    k_seg_sort(const U* data_in, U* data, U* __restrict__ alt, const unsigned long long* __restrict__ offsets,
               const unsigned int* __restrict__ lists, size_t n_seg, const SegPlan* __restrict__ plan,
               unsigned int* __restrict__ counter, SegMethods methods) {
    static_assert(SegSmem::bytes<U>() <= (size_t)MSD_SMEM, "the on-chip sorts' areas fit the launch's shared memory");
    extern __shared__ __align__(128) unsigned char smem[];
    U* sm = reinterpret_cast<U*>(smem);
    uint32_t* cnt = reinterpret_cast<uint32_t*>(smem + SegSmem::cnt_off<U>());
    int* misc = reinterpret_cast<int*>(smem + SegSmem::misc_off<U>());
    int* warp_tot = misc;                                            // [32]
    unsigned long long* red = reinterpret_cast<unsigned long long*>(misc + 32);
    int* item_s = misc + 40;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned int items = plan->items;
    // thread 0 holds the claim on the CTA's next item and brings a single
    // segment's keys into L2 while this item is sorted (the sorts run from
    // shared memory and L2, so their first read no longer waits on DRAM)
    unsigned int next = 0;
    if (threadIdx.x == 0) next = atomicAdd(counter, 1u);
    for (;;) {
        if (threadIdx.x == 0) {
            *item_s = (int)next;
            next = atomicAdd(counter, 1u);
            if (next < items) {
                int nbin;
                unsigned int nfirst;
                seg_item(*plan, next, &nbin, &nfirst);
                if (nbin != SEG_BIN_WARP && !(nbin < SEG_BLOCK_BINS && seg_grouped(nbin, methods.m[nbin]))) {
                    const unsigned int s = lists[(size_t)nbin * n_seg + nfirst];
                    const unsigned long long b = offsets[s];
                    const unsigned long long e = min(offsets[s + 1], b + (1ull << 22));  // at most 16-32 MB
                    prefetch_l2(data_in + b, data_in + e);
                }
            }
        }
        __syncthreads();
        const unsigned int item = (unsigned int)*item_s;
        __syncthreads();
        if (item >= items) break;
        int bin;
        unsigned int first;
        seg_item(*plan, item, &bin, &first);
        if (bin == SEG_BIN_WARP) {
            const unsigned int idx = first + warp;
            if (idx < plan->count[SEG_BIN_WARP]) {
                const unsigned int s = lists[(size_t)SEG_BIN_WARP * n_seg + idx];
                const unsigned long long b = offsets[s];
                seg_warp_sort<U, XF>(data_in + b, data + b, (int)(offsets[s + 1] - b), lane);
            }
        } else if (bin < SEG_BLOCK_BINS && methods.m[bin] == SEG_MSD_GROUPS) {
            if constexpr (sizeof(U) >= 4) {
                auto run = [&](auto g_tag) {
                    constexpr int G = decltype(g_tag)::value;
                    const int g = threadIdx.x / G;
                    const unsigned int idx = first + (unsigned int)g;
                    if (idx < plan->count[bin]) {
                        const unsigned int s = lists[(size_t)bin * n_seg + idx];
                        const unsigned long long b = offsets[s];
                        msd_group<U, XF, G>(data_in + b, data + b, (int)(offsets[s + 1] - b),
                                            smem + (size_t)g * SegGroup<U, G>::slice, 1 + g);
                    }
                };
                if (bin == 2) run(std::integral_constant<int, 256>{});
                else run(std::integral_constant<int, 512>{});
            }
        } else if (bin < SEG_BLOCK_BINS && seg_grouped(bin, methods.m[bin])) {
            const unsigned int idx = first + warp;
            if (idx < plan->count[bin]) {
                const unsigned int s = lists[(size_t)bin * n_seg + idx];
                const unsigned long long b = offsets[s];
                const int len = (int)(offsets[s + 1] - b);
                if (bin == 0 || len <= 512) {
                    if (bin == 0) warp_bitonic<U, XF, 8>(data_in + b, data + b, len, lane);
                    else warp_bitonic<U, XF, 16>(data_in + b, data + b, len, lane);
                } else if constexpr (sizeof(U) <= 4) {
                    warp_bitonic<U, XF, 32>(data_in + b, data + b, len, lane);
                }
            }
        } else {
            const unsigned int s = lists[(size_t)bin * n_seg + first];
            const unsigned long long b = offsets[s];
            const int len = (int)(offsets[s + 1] - b);
            if (bin == SEG_BIN_LARGE) {
                if constexpr (sizeof(U) >= 4) {
                    msd_sort<U, XF>(data_in + b, data + b, alt + b, len, smem);
                } else {  // 8- and 16-bit keys crowd the sub-ranges: straight to the CTA-level LSD
                    uint32_t* hist = reinterpret_cast<uint32_t*>(smem + SegSmem::hist_off<U>());
                    uint32_t* run = reinterpret_cast<uint32_t*>(smem + SegSmem::run_off<U>());
                    seg_large_sort<U, XF>(data_in + b, data + b, alt + b, len, sm, cnt, warp_tot, red, hist, run,
                                          run + 256, run + 512);
                }
            } else {
                const int m = methods.m[bin];
                if (m == SEG_MSD) {
                    if constexpr (sizeof(U) >= 4) msd_sort<U, XF>(data_in + b, data + b, alt + b, len, smem);
                    else seg_block_radix<U, XF, 8>(data_in + b, data + b, len, sm, cnt, warp_tot, red);
                } else if (m == SEG_BITONIC) seg_block_bitonic<U, XF>(data_in + b, data + b, len, sm);
                else if (m == SEG_RADIX4) seg_block_radix<U, XF, 4>(data_in + b, data + b, len, sm, cnt, warp_tot, red);
                else seg_block_radix<U, XF, 8>(data_in + b, data + b, len, sm, cnt, warp_tot, red);
            }
        }
        __syncthreads();
    }
}

}  // namespace ts
