// ts_lsd.cuh — the LSD radix sort kernels.
//
//   k_scan      one read (early exit): bits that vary (src/radix/histogram.rs:55-68)
//               and whether the input is already sorted either way
//               (src/presorted.rs:15-65)
//   k_hist      one read: histograms of every varying digit
//               (src/radix/histogram.rs:15-110)
//   k_plan      live passes (src/radix/mod.rs:229-239) and the exclusive scans
//               (src/radix/prefix_sum.rs:17-24), decided on the device
//   k_onesweep  one stable scatter pass per live digit
//               (src/radix/scatter.rs:26-247): warp ranking with match.any,
//               decoupled look-back across tiles, the tile reordered in shared
//               memory so that global writes are runs per digit. The key
//               transform (src/key.rs:135-197) is fused into the first load
//               and the last store. Optionally carries a u32 position (the
//               stable order() of src/by_key.rs:254-310).
//   k_finish    copy-back for an odd pass count (src/radix/mod.rs:265-267),
//               the reversal of descending input, iota for an order that
//               needed no pass
#pragma once

#include "ts_common.cuh"

namespace ts {

template <typename U>
struct Vec16 {
    static constexpr int N = 16 / sizeof(U);
    union {
        uint4 v;
        U e[N];
    };
};

__device__ __forceinline__ bool all_digits_vary(unsigned long long diff, int bits, int nd) {
    const unsigned long long mask = (1ull << bits) - 1;
    bool all = true;
    for (int d = 0; d < nd; ++d) all &= ((diff >> (d * bits)) & mask) != 0;
    return all;
}

// ---------------------------------------------------------------------------
// k_scan: OR of (key ^ first key) and the two sortedness flags. Warps leave
// as soon as every digit has varied and both directions are disproved,
// which random input does in its first chunk.
// ---------------------------------------------------------------------------
template <typename U, int XF, int THREADS>
__global__ void __launch_bounds__(THREADS) k_scan(const U* __restrict__ src, size_t n, int bits, int nd,
                                                  ScanState* __restrict__ st, int vec_ok) {
    using V = Vec16<U>;
    constexpr int VN = V::N;
    constexpr int UNROLL = 4;
    const U first = to_key<U, XF>(src[0]);
    const int lane = threadIdx.x & 31;
    unsigned long long diff = 0, published = 0;
    unsigned flags = 0, pub_flags = 0;
    const size_t per_iter = (size_t)THREADS * VN * UNROLL;
    for (size_t it = (size_t)blockIdx.x * per_iter; it < n; it += (size_t)gridDim.x * per_iter) {
#pragma unroll
        for (int u = 0; u < UNROLL; ++u) {
            const size_t base = it + ((size_t)u * THREADS + threadIdx.x) * VN;
            U k[VN];
            if (vec_ok && base + VN <= n) {
                V x;
                x.v = __ldcs(reinterpret_cast<const uint4*>(src + base));
#pragma unroll
                for (int e = 0; e < VN; ++e) k[e] = x.e[e];
            } else {
#pragma unroll
                for (int e = 0; e < VN; ++e) k[e] = base + e < n ? src[base + e] : src[n - 1];
            }
#pragma unroll
            for (int e = 0; e < VN; ++e) k[e] = to_key<U, XF>(k[e]);
            // the element just before this thread's vector
            U prev = __shfl_up_sync(0xffffffffu, k[VN - 1], 1);
            if (lane == 0) prev = base > 0 && base - 1 < n ? to_key<U, XF>(src[base - 1]) : k[0];
            if (base < n) {
                if (base > 0) {
                    flags |= prev > k[0] ? SCAN_NOT_ASC : 0u;
                    flags |= prev < k[0] ? SCAN_NOT_DESC : 0u;
                }
#pragma unroll
                for (int e = 0; e < VN; ++e) {
                    if (base + e < n) {
                        diff |= (unsigned long long)(k[e] ^ first);
                        if (e > 0) {
                            flags |= k[e - 1] > k[e] ? SCAN_NOT_ASC : 0u;
                            flags |= k[e - 1] < k[e] ? SCAN_NOT_DESC : 0u;
                        }
                    }
                }
            }
        }
        // warp-level merge, publish what is new, and read the global state
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            diff |= __shfl_xor_sync(0xffffffffu, diff, o);
            flags |= __shfl_xor_sync(0xffffffffu, flags, o);
        }
        int stop = 0;
        if (lane == 0) {
            if (diff & ~published) {
                atomicOr(&st->diff, diff);
                published |= diff;
            }
            if (flags & ~pub_flags) {
                atomicOr(&st->flags, flags);
                pub_flags |= flags;
            }
            unsigned long long g = ld_volatile_u64(&st->diff);
            unsigned gf = ld_volatile_u32(&st->flags);
            stop = (gf == (SCAN_NOT_ASC | SCAN_NOT_DESC)) && all_digits_vary(g, bits, nd);
        }
        if (__shfl_sync(0xffffffffu, stop, 0)) return;
    }
}

// ---------------------------------------------------------------------------
// k_hist: histograms of the varying digits in one read. Sub-histograms per
// (lane % COPIES) keep lanes that share a digit off one address; the copy
// index is the fastest-moving so those lanes also sit in different banks.
// ---------------------------------------------------------------------------
template <typename U, int XF, int BITS, int THREADS>
__global__ void __launch_bounds__(THREADS) k_hist(const U* __restrict__ src, size_t n, const ScanState* __restrict__ st,
                                                  unsigned long long* __restrict__ ghist, int vec_ok) {
    constexpr int RADIX = 1 << BITS;
    constexpr int ND = (Bits<U>::W + BITS - 1) / BITS;
    constexpr int COPIES = RADIX <= 256 ? 4 : 1;
    using V = Vec16<U>;
    constexpr int VN = V::N;
    constexpr int UNROLL = 2;
    extern __shared__ __align__(16) uint32_t h_s[];  // [ND][RADIX][COPIES]
    const unsigned long long diff = st->diff;
    uint32_t counted = 0;
#pragma unroll
    for (int d = 0; d < ND; ++d)
        if ((diff >> (d * BITS)) & (unsigned long long)(RADIX - 1)) counted |= 1u << d;
    for (int i = threadIdx.x; i < ND * RADIX * COPIES; i += THREADS) h_s[i] = 0;
    __syncthreads();
    const int copy = threadIdx.x % COPIES;
    const size_t per_iter = (size_t)THREADS * VN * UNROLL;
    for (size_t it = (size_t)blockIdx.x * per_iter; it < n; it += (size_t)gridDim.x * per_iter) {
#pragma unroll
        for (int u = 0; u < UNROLL; ++u) {
            const size_t base = it + ((size_t)u * THREADS + threadIdx.x) * VN;
            if (base >= n) break;
            U k[VN];
            int cnt = VN;
            if (vec_ok && base + VN <= n) {
                V x;
                x.v = __ldcs(reinterpret_cast<const uint4*>(src + base));
#pragma unroll
                for (int e = 0; e < VN; ++e) k[e] = x.e[e];
            } else {
                cnt = (int)min((size_t)VN, n - base);
#pragma unroll
                for (int e = 0; e < VN; ++e) k[e] = e < cnt ? src[base + e] : (U)0;
            }
#pragma unroll
            for (int e = 0; e < VN; ++e) {
                if (e < cnt) {
                    const U key = to_key<U, XF>(k[e]);
#pragma unroll
                    for (int d = 0; d < ND; ++d)
                        if (counted & (1u << d))
                            atomicAdd(&h_s[(d * RADIX + digit_of(key, d * BITS, RADIX - 1)) * COPIES + copy], 1u);
                }
            }
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < ND * RADIX; i += THREADS) {
        uint32_t s = 0;
#pragma unroll
        for (int c = 0; c < COPIES; ++c) s += h_s[i * COPIES + c];
        if (s) atomicAdd(&ghist[i], (unsigned long long)s);
    }
}

// ---------------------------------------------------------------------------
// k_plan: one CTA. Live passes are the counted digits whose histogram does
// not hold every key in the first key's bucket; each gets its exclusive scan.
// `stable` (sort_by_key) leaves descending input to the passes, since a
// plain reversal would reverse equal keys.
// ---------------------------------------------------------------------------
template <typename U, int XF, int BITS>
__global__ void __launch_bounds__(1024) k_plan(const U* __restrict__ src, size_t n, const ScanState* __restrict__ st,
                                               const unsigned long long* __restrict__ ghist,
                                               unsigned long long* __restrict__ bins, Plan* __restrict__ plan,
                                               int stable) {
    constexpr int RADIX = 1 << BITS;
    constexpr int ND = (Bits<U>::W + BITS - 1) / BITS;
    __shared__ int live_s[ND];
    const U first = to_key<U, XF>(src[0]);
    const unsigned long long diff = st->diff;
    if (threadIdx.x < ND) {
        const int d = threadIdx.x;
        const bool counted = ((diff >> (d * BITS)) & (unsigned long long)(RADIX - 1)) != 0;
        live_s[d] = counted && ghist[(size_t)d * RADIX + digit_of(first, d * BITS, RADIX - 1)] < n;
    }
    __syncthreads();
    // warp w scans digit w's histogram
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp < ND && live_s[warp]) {
        unsigned long long carry = 0;
        for (int r0 = 0; r0 < RADIX; r0 += 32) {
            const int r = r0 + lane;
            unsigned long long v = r < RADIX ? ghist[(size_t)warp * RADIX + r] : 0ull;
            unsigned long long x = v;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            if (r < RADIX) bins[(size_t)warp * RADIX + r] = carry + x - v;
            carry += __shfl_sync(0xffffffffu, x, 31);
        }
    }
    if (threadIdx.x == 0) {
        const unsigned f = st->flags;
        int mode = MODE_SORT;
        if (!(f & SCAN_NOT_ASC)) mode = MODE_SORTED;
        else if (!stable && !(f & SCAN_NOT_DESC)) mode = MODE_REVERSE;
        int m = 0;
        if (mode == MODE_SORT)
            for (int d = 0; d < ND; ++d)
                if (live_s[d]) plan->pass[m++] = d;
        plan->n_live = m;
        plan->mode = mode;
    }
}

// ---------------------------------------------------------------------------
// k_onesweep: one live digit pass. Persistent CTAs take tiles in order from a
// counter, so a tile only ever waits on tiles already taken by running CTAs.
// ---------------------------------------------------------------------------
template <typename U, bool PAIRS>
struct SweepArgs {
    const U* in;                 // slot 0 source
    U* pp[2];                    // ping-pong: slot j writes pp[j & 1], reads pp[(j - 1) & 1]
    const uint32_t* vin;         // unused: slot 0 starts from positions 0..n-1
    uint32_t* vpp[2];            // position ping-pong (PAIRS)
    uint32_t* vout;              // last slot's positions: the order (PAIRS)
    size_t n;                    // keys in the whole sort
    size_t portion_begin;        // first key of this launch's portion
    int portion_tiles;           // tiles in this portion
    int slot;                    // which live pass this launch is
    int write_keys_last;         // PAIRS: does the last pass write keys too
    const Plan* plan;
    const unsigned long long* bins;   // [ND][RADIX] exclusive scans
    const unsigned long long* carry_in;  // [RADIX] keys of this digit in earlier portions, or null
    unsigned long long* carry_out;       // written by the portion's last tile, or null
    uint32_t* lookback;          // [portion_tiles][RADIX], zero when the launch starts
    uint32_t* lookback_next;     // the next launch's region: this launch zeroes it
    size_t lookback_words;       // words per region (a multiple of 4)
    uint32_t* tile_counter;      // zeroed before the launch
    uint32_t* error;
};

template <typename U, int BITS, int THREADS, int IPT, bool PAIRS>
struct SweepSmem {
    static constexpr int RADIX = 1 << BITS;
    static constexpr int TILE = THREADS * IPT;
    static constexpr int WARPS = THREADS / 32;
    using CT = typename std::conditional<(RADIX > 256), uint16_t, uint32_t>::type;
    static constexpr size_t keys_off = 0;
    static constexpr size_t vals_off = (keys_off + sizeof(U) * TILE + 15) / 16 * 16;
    static constexpr size_t cnt_off = (vals_off + (PAIRS ? 4 * TILE : 0) + 15) / 16 * 16;
    static constexpr size_t gbase_off = (cnt_off + sizeof(CT) * WARPS * RADIX + 15) / 16 * 16;
    static constexpr size_t misc_off = gbase_off + 8 * RADIX;
    static constexpr size_t bytes = misc_off + 4 * 64;
};

template <typename U, int XF, int BITS, int THREADS, int IPT, bool PAIRS>
__global__ void __launch_bounds__(THREADS, 2) k_onesweep(SweepArgs<U, PAIRS> a) {
    using L = SweepSmem<U, BITS, THREADS, IPT, PAIRS>;
    using CT = typename L::CT;
    constexpr int RADIX = L::RADIX;
    constexpr int TILE = L::TILE;
    constexpr int WARPS = L::WARPS;
    constexpr uint32_t MASK = RADIX - 1;
    constexpr int DPT = RADIX >= THREADS ? RADIX / THREADS : 1;   // digits per owner thread
    constexpr int OWNERS = RADIX / DPT;
    static_assert(TILE < 65536 || RADIX <= 256, "16-bit counters need tiles below 65536 keys");
    static_assert(RADIX % DPT == 0 && OWNERS <= THREADS, "digit ownership");

    const int mode = a.plan->mode, n_live = a.plan->n_live;
    if (mode != MODE_SORT || a.slot >= n_live) return;
    const int pass = a.plan->pass[a.slot];
    const int shift = pass * BITS;
    const bool first = a.slot == 0;
    const bool last = a.slot == n_live - 1;
    const U* __restrict__ src = first ? a.in : a.pp[(a.slot - 1) & 1];
    U* __restrict__ dst = a.pp[a.slot & 1];
    const uint32_t* __restrict__ vsrc = first ? nullptr : a.vpp[(a.slot - 1) & 1];
    uint32_t* __restrict__ vdst = last ? a.vout : a.vpp[a.slot & 1];
    const bool write_keys = !PAIRS || !last || a.write_keys_last;
    const unsigned long long* __restrict__ bins = a.bins + (size_t)pass * RADIX;

    extern __shared__ __align__(16) unsigned char smem[];
    U* keys_s = reinterpret_cast<U*>(smem + L::keys_off);
    uint32_t* vals_s = reinterpret_cast<uint32_t*>(smem + L::vals_off);
    CT* cnt_s = reinterpret_cast<CT*>(smem + L::cnt_off);
    long long* gbase_s = reinterpret_cast<long long*>(smem + L::gbase_off);
    int* misc_s = reinterpret_cast<int*>(smem + L::misc_off);  // [0] tile, [32..] warp totals

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const size_t portion_end = min(a.n, a.portion_begin + (size_t)a.portion_tiles * TILE);

    // The previous launch used the other region; clear it for the next one.
    {
        uint4* z = reinterpret_cast<uint4*>(a.lookback_next);
        const size_t nz = a.lookback_words / 4;
        for (size_t i = (size_t)blockIdx.x * THREADS + tid; i < nz; i += (size_t)gridDim.x * THREADS)
            z[i] = make_uint4(0u, 0u, 0u, 0u);
    }

    for (;;) {
        if (tid == 0) misc_s[0] = (int)atomicAdd(a.tile_counter, 1u);
        __syncthreads();
        const int t = misc_s[0];
        if (t >= a.portion_tiles) break;
        const size_t tile_base = a.portion_begin + (size_t)t * TILE;
        const int tile_n = (int)min((size_t)TILE, portion_end - tile_base);

        for (int i = tid; i < WARPS * RADIX; i += THREADS) cnt_s[i] = 0;

        // ---- load: warp-striped, item i of lane l is tile index w*32*IPT + i*32 + l
        U k[IPT];
        uint32_t v[IPT];
        const int wbase = warp * 32 * IPT + lane;
#pragma unroll
        for (int i = 0; i < IPT; ++i) {
            const int idx = wbase + i * 32;
            if (idx < tile_n) {
                k[i] = __ldcs(src + tile_base + idx);
                if constexpr (PAIRS) v[i] = first ? (uint32_t)(tile_base + idx) : __ldcs(vsrc + tile_base + idx);
            } else {
                k[i] = 0;
                if constexpr (PAIRS) v[i] = 0;
            }
        }
        if (first) {
#pragma unroll
            for (int i = 0; i < IPT; ++i) k[i] = to_key<U, XF>(k[i]);
        }
        __syncthreads();

        // ---- rank inside the warp: stable, one match.any per item
        CT* my_cnt = cnt_s + warp * RADIX;
        uint32_t rank[IPT];
        const uint32_t lt = lanemask_lt();
#pragma unroll
        for (int i = 0; i < IPT; ++i) {
            const bool valid = wbase + i * 32 < tile_n;
            const uint32_t d = valid ? digit_of(k[i], shift, MASK) : (uint32_t)RADIX;
            const uint32_t peers = __match_any_sync(0xffffffffu, d);
            const uint32_t leader = 31 - __clz(peers);
            uint32_t c = 0;
            if (valid) c = my_cnt[d];
            __syncwarp();
            if (valid && lane == (int)leader) my_cnt[d] = (CT)(c + __popc(peers));
            __syncwarp();
            rank[i] = c + __popc(peers & lt);
        }
        __syncthreads();

        // ---- per digit: prefix over warps, tile count, publish, tile-local start
        uint32_t tcount[DPT];
        if (tid < OWNERS) {
#pragma unroll
            for (int q = 0; q < DPT; ++q) {
                const int r = tid * DPT + q;
                uint32_t s = 0;
#pragma unroll 4
                for (int w = 0; w < WARPS; ++w) {
                    const uint32_t c = cnt_s[w * RADIX + r];
                    cnt_s[w * RADIX + r] = (CT)s;
                    s += c;
                }
                tcount[q] = s;
                st_relaxed_gpu(a.lookback + (size_t)t * RADIX + r, (t == 0 ? LB_FLAG_INC : LB_FLAG_AGG) | s);
            }
        }
        // block exclusive scan of the tile counts over digits (owners only hold data)
        uint32_t own = 0;
        if (tid < OWNERS) {
#pragma unroll
            for (int q = 0; q < DPT; ++q) own += tcount[q];
        }
        uint32_t x = own;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) misc_s[32 + warp] = (int)x;
        __syncthreads();
        if (warp == 0) {
            uint32_t wt = lane < WARPS ? (uint32_t)misc_s[32 + lane] : 0u;
            uint32_t z = wt;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, z, o);
                if (lane >= o) z += y;
            }
            if (lane < WARPS) misc_s[32 + lane] = (int)(z - wt);
        }
        __syncthreads();
        uint32_t lstart[DPT];
        if (tid < OWNERS) {
            uint32_t run = (uint32_t)misc_s[32 + warp] + x - own;
#pragma unroll
            for (int q = 0; q < DPT; ++q) {
                lstart[q] = run;
                run += tcount[q];
                const int r = tid * DPT + q;
#pragma unroll 4
                for (int w = 0; w < WARPS; ++w) cnt_s[w * RADIX + r] = (CT)(cnt_s[w * RADIX + r] + lstart[q]);
            }
        }
        __syncthreads();

        // ---- reorder the tile in shared memory by digit
#pragma unroll
        for (int i = 0; i < IPT; ++i) {
            if (wbase + i * 32 < tile_n) {
                const uint32_t d = digit_of(k[i], shift, MASK);
                const uint32_t pos = (uint32_t)my_cnt[d] + rank[i];
                if (pos < (uint32_t)TILE) {
                    keys_s[pos] = k[i];
                    if constexpr (PAIRS) vals_s[pos] = v[i];
                } else {
                    atomicOr(a.error, ERR_BOUNDS);
                }
            }
        }

        // ---- decoupled look-back: keys of each digit in earlier tiles
        if (tid < OWNERS) {
#pragma unroll
            for (int q = 0; q < DPT; ++q) {
                const int r = tid * DPT + q;
                uint32_t excl = 0;
                if (t > 0) {
                    int j = t - 1;
                    uint32_t spins = 0;
                    while (j >= 0) {
                        const uint32_t w = ld_relaxed_gpu(a.lookback + (size_t)j * RADIX + r);
                        const uint32_t f = w & ~LB_VALUE;
                        if (f == 0) {
                            if (++spins > SPIN_LIMIT) {
                                atomicOr(a.error, ERR_TIMEOUT);
                                break;
                            }
                            continue;
                        }
                        excl += w & LB_VALUE;
                        if (f == LB_FLAG_INC) break;
                        --j;
                    }
                    st_relaxed_gpu(a.lookback + (size_t)t * RADIX + r, LB_FLAG_INC | (excl + tcount[q]));
                }
                const unsigned long long carry = a.carry_in ? a.carry_in[r] : 0ull;
                gbase_s[r] = (long long)(bins[r] + carry + excl) - (long long)lstart[q];
                if (a.carry_out && t == a.portion_tiles - 1) a.carry_out[r] = carry + excl + tcount[q];
            }
        }
        __syncthreads();

        // ---- write runs per digit: consecutive threads, consecutive addresses
#pragma unroll
        for (int i = 0; i < IPT; ++i) {
            const int s = i * THREADS + tid;
            if (s < tile_n) {
                const U key = keys_s[s];
                const uint32_t d = digit_of(key, shift, MASK);
                const unsigned long long pos = (unsigned long long)(gbase_s[d] + s);
                if (pos < a.n) {
                    if (write_keys) dst[pos] = last ? from_key<U, XF>(key) : key;
                    if constexpr (PAIRS) vdst[pos] = vals_s[s];
                } else {
                    atomicOr(a.error, ERR_BOUNDS);
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Finishing kernels, each a no-op unless the plan calls for it.
// ---------------------------------------------------------------------------
template <typename U>
__global__ void k_copy_back(const Plan* __restrict__ plan, const U* __restrict__ from, U* __restrict__ to, size_t n,
                            int vec_ok) {
    if (plan->mode != MODE_SORT || (plan->n_live & 1) == 0) return;
    using V = Vec16<U>;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    if (vec_ok) {
        const size_t nv = n / V::N;
        const uint4* f = reinterpret_cast<const uint4*>(from);
        uint4* o = reinterpret_cast<uint4*>(to);
        for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += stride) __stcs(o + i, __ldcs(f + i));
        for (size_t i = nv * V::N + (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) to[i] = from[i];
    } else {
        for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) to[i] = from[i];
    }
}

template <typename U>
__global__ void k_reverse(const Plan* __restrict__ plan, U* __restrict__ data, size_t n) {
    if (plan->mode != MODE_REVERSE) return;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n / 2; i += stride) {
        const U x = data[i];
        data[i] = data[n - 1 - i];
        data[n - 1 - i] = x;
    }
}

static __global__ void k_iota_if_unsorted(const Plan* __restrict__ plan, uint32_t* __restrict__ order, size_t n) {
    if (plan->mode == MODE_SORT && plan->n_live > 0) return;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) order[i] = (uint32_t)i;
}

}  // namespace ts
