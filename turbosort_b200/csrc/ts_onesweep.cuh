// ts_onesweep.cuh — one stable LSD scatter pass (src/radix/scatter.rs:26-247)
// per launch, as a decoupled-look-back "onesweep" over tiles of keys.
//
// Per tile (THREADS x IPT keys), in a persistent CTA that takes tiles in
// order from a counter:
//   1. the keys arrive in shared memory by one bulk copy (cp.async.bulk, no
//      multicast); with two buffers (NBUF = 2) it is issued one tile ahead,
//      with one the CTA claims its next tile early, prefetches it into L2,
//      and issues its copy as soon as this tile's keys are staged (step 4);
//   2. a counting pass builds per-warp digit counts, the tile's
//      digit counts are published to the look-back array at once, and the
//      tile-local start of every (digit, warp) run is scanned;
//   3. a ranking pass finds each key's equals inside its warp (one ballot per
//      digit bit, or match.any for some items) and writes the key straight to
//      its sorted place in a shared staging tile (stable: warp order, then
//      item order, then lane);
//   4. the digit owners finish the look-back (keys of their digit in all
//      earlier tiles), a few predecessors per round trip;
//   5. the staged tile goes out as runs per digit: consecutive threads write
//      consecutive addresses.
// The key transform (src/key.rs:135-197) is applied as the first pass reads
// and undone as the last pass writes. With PAIRS a u32 position travels with
// each key (the stable order() of src/by_key.rs:254-310); the first pass
// makes the positions itself.
#pragma once

#include <type_traits>

#include "ts_common.cuh"

namespace ts {

template <typename U, bool PAIRS>
struct SweepArgs {
    const U* in;                 // slot 0 source
    U* pp[2];                    // ping-pong: slot j writes pp[j & 1], reads pp[(j - 1) & 1]
    uint32_t* vpp[2];            // position ping-pong (PAIRS)
    uint32_t* vout;              // last slot's positions: the order (PAIRS)
    size_t n;                    // keys in the whole sort
    size_t portion_begin;        // first key of this launch's portion
    int portion_tiles;           // tiles in this portion
    int slot;                    // which live pass this launch is
    int write_keys_last;         // PAIRS: does the last pass write keys too
    const Plan* plan;
    const unsigned long long* bins;      // [ND][RADIX] exclusive scans
    const unsigned long long* carry_in;  // [RADIX] keys of this digit in earlier portions, or null
    unsigned long long* carry_out;       // written by the portion's last tile, or null
    uint32_t* lookback;          // [portion_tiles][RADIX], zero when the launch starts
    uint32_t* lookback_next;     // the next launch's region: this launch zeroes it
    size_t lookback_words;       // words per region (a multiple of 4)
    uint32_t* tile_counter;      // zeroed before the launch
    uint32_t* error;
    uint32_t spin_limit;         // look-back rounds without progress before ERR_TIMEOUT
    int withhold_tile0;          // test hook: tile 0 never publishes (its successors' waits run out)
};

// LBC: the region of each digit's tile count and start that the paired
// look-back (LB_PAIR) reads; left out otherwise.
template <typename U, int BITS, int THREADS, int IPT, bool PAIRS, int NBUF, bool LBC>
struct SweepSmem {
    static constexpr int RADIX = 1 << BITS;
    static constexpr int WARPS = THREADS / 32;
    static constexpr int RANK_WARPS = WARPS;
    static constexpr int TILE = RANK_WARPS * 32 * IPT;
    static constexpr size_t al(size_t x) { return (x + 127) / 128 * 128; }
    static constexpr size_t kbuf_off = 0;                                             // [NBUF][TILE] U
    static constexpr size_t vbuf_off = al(kbuf_off + (size_t)NBUF * TILE * sizeof(U));  // [NBUF][TILE] u32
    static constexpr size_t sk_off = al(vbuf_off + (PAIRS ? (size_t)NBUF * TILE * 4 : 0));  // [TILE] U sorted
    static constexpr size_t sv_off = al(sk_off + (size_t)TILE * sizeof(U));           // [TILE] u32 sorted
    static constexpr size_t cnt_off = al(sv_off + (PAIRS ? (size_t)TILE * 4 : 0));    // [RANK_WARPS][RADIX] u32
    static constexpr size_t gbase_off = al(cnt_off + (size_t)RANK_WARPS * RADIX * 4);  // [RADIX] i64
    static constexpr size_t lbc_off = al(gbase_off + (size_t)RADIX * 8);              // [RADIX] u32 x2: counts, starts
    static constexpr size_t bar_off = al(lbc_off + (LBC ? (size_t)RADIX * 8 : 0));     // [2] mbarrier
    static constexpr size_t misc_off = bar_off + 16;                                  // ints
    static constexpr size_t bytes = misc_off + 4 * 64;
    static_assert(TILE * sizeof(U) % 16 == 0, "bulk copies move multiples of 16 bytes");
};

__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// The lanes of a warp whose BITS-bit digit equals this lane's. One ballot per
// digit bit gives the warp's bit-planes; the digit's bits are taken in
// groups of up to five, and for each group lane L builds the entry of a
// small table for the group value L stands for (the lanes whose bits in the
// group equal L's index); each lane then reads its own digit's entry of every
// table with a shuffle and ANDs them. x[b] holds, per lane, all ones where
// the lane's index has bit (b mod 5) clear (set up once by init). 8-bit
// digits take two tables (5 + 3 bits), 11-bit ones three (5 + 5 + 1).
template <int BITS>
struct PeerMasks {
    static_assert(BITS >= 1 && BITS <= 15, "three lookup tables cover digits of up to 15 bits");
    static constexpr int NT = (BITS + 4) / 5;  // tables
    uint32_t x[BITS];
    __device__ __forceinline__ void init(int lane) {
#pragma unroll
        for (int b = 0; b < BITS; ++b) x[b] = ((lane >> (b % 5)) & 1) ? 0u : 0xffffffffu;
    }
    __device__ __forceinline__ uint32_t peers(uint32_t d) const {
        uint32_t tbl[NT];
#pragma unroll
        for (int t = 0; t < NT; ++t) tbl[t] = 0xffffffffu;
#pragma unroll
        for (int b = 0; b < BITS; ++b) tbl[b / 5] &= __ballot_sync(0xffffffffu, (d >> b) & 1u) ^ x[b];
        uint32_t p = 0xffffffffu;
#pragma unroll
        for (int t = 0; t < NT; ++t) {
            const int w = BITS - 5 * t < 5 ? BITS - 5 * t : 5;
            p &= __shfl_sync(0xffffffffu, tbl[t], (int)((d >> (5 * t)) & ((1u << w) - 1)));
        }
        return p;
    }
};

// D consecutive per-warp counters of one owner thread, moved as one word
// (D = 1, 2 or 4; the address is D-word aligned).
template <int D>
__device__ __forceinline__ void cnt_load(const uint32_t* p, uint32_t (&v)[D]) {
    static_assert(D == 1 || D == 2 || D == 4, "digits per owner");
    if constexpr (D == 4) {
        const uint4 x = *reinterpret_cast<const uint4*>(p);
        v[0] = x.x, v[1] = x.y, v[2] = x.z, v[3] = x.w;
    } else if constexpr (D == 2) {
        const uint2 x = *reinterpret_cast<const uint2*>(p);
        v[0] = x.x, v[1] = x.y;
    } else {
        v[0] = *p;
    }
}
template <int D>
__device__ __forceinline__ void cnt_store(uint32_t* p, const uint32_t (&v)[D]) {
    if constexpr (D == 4) *reinterpret_cast<uint4*>(p) = make_uint4(v[0], v[1], v[2], v[3]);
    else if constexpr (D == 2) *reinterpret_cast<uint2*>(p) = make_uint2(v[0], v[1]);
    else *p = v[0];
}
// WORDS counters (a multiple of 4, 16-byte aligned) set to zero, 16 bytes a store
template <int WORDS, int THREADS>
__device__ __forceinline__ void zero_counters(uint32_t* cnt, int tid) {
    static_assert(WORDS % 4 == 0, "whole 16-byte words");
    uint4* z = reinterpret_cast<uint4*>(cnt);
#pragma unroll
    for (int i = tid; i < WORDS / 4; i += THREADS) z[i] = make_uint4(0u, 0u, 0u, 0u);
}

// Items i with i % MATCH_MOD < MATCH_CNT find their equal digits with the
// match.any instruction, which runs on a different pipe from the ballots; the
// rest use PeerMasks. The split keeps both pipes busy.
//
// UNSTABLE1: the first live pass of a keys-only sort ranks with one shared
// atomic per key instead of finding its equals. That pass has no input
// order to keep: after it the keys need only be ordered by its digit, and
// the later (stable) passes order keys of equal higher digits by it. Keys
// equal in every bit are the same bit pattern, so their order is not
// observable. With positions (PAIRS) every pass stays stable.
template <typename U, int XF, int BITS, int THREADS, int IPT, bool PAIRS, int NBUF, bool BIG, int MATCH_MOD,
          int MATCH_CNT, bool UNSTABLE1 = false, bool RANK_AHEAD = false, int LBW = LB_WINDOW, bool LB_PAIR = false>
__global__ void __launch_bounds__(THREADS, SweepSmem<U, BITS, THREADS, IPT, PAIRS, NBUF, LB_PAIR>::bytes <= 113 * 1024
                                               ? 1024 / THREADS
                                               : 1) k_onesweep(SweepArgs<U, PAIRS> a) {
    dep_wait();
    dep_release();
    using L = SweepSmem<U, BITS, THREADS, IPT, PAIRS, NBUF, LB_PAIR>;
    using OFF = typename std::conditional<BIG, long long, int>::type;
    constexpr int RADIX = L::RADIX;
    constexpr int TILE = L::TILE;
    constexpr int RANK_WARPS = L::RANK_WARPS;
    constexpr uint32_t MASK = RADIX - 1;
    constexpr int OWNERS = RADIX < THREADS ? RADIX : THREADS;  // threads that own digits
    constexpr int DPT = RADIX / OWNERS;                          // digits per owner thread
    constexpr int OWNER_WARPS = (OWNERS + 31) / 32;
    constexpr int SCATTER_IT = (TILE + THREADS - 1) / THREADS;
    static_assert(RADIX % OWNERS == 0 && OWNER_WARPS <= RANK_WARPS, "digit ownership");

    const int mode = a.plan->mode, n_live = a.plan->n_live;
    if (mode != MODE_SORT || a.slot >= n_live) return;
    const int pass = a.plan->pass[a.slot];
    const int shift = pass * BITS;
    const bool first = a.slot == 0;
    const bool last = a.slot == n_live - 1;
    const U* __restrict__ src = first ? a.in : a.pp[(a.slot - 1) & 1];
    U* __restrict__ dst = a.pp[a.slot & 1];
    const uint32_t* __restrict__ vsrc = (PAIRS && !first) ? a.vpp[(a.slot - 1) & 1] : nullptr;
    uint32_t* __restrict__ vdst = last ? a.vout : a.vpp[a.slot & 1];
    const bool write_keys = !PAIRS || !last || a.write_keys_last;
    const unsigned long long* __restrict__ bins = a.bins + (size_t)pass * RADIX;

    extern __shared__ __align__(128) unsigned char smem[];
    U* kbuf = reinterpret_cast<U*>(smem + L::kbuf_off);
    uint32_t* vbuf = reinterpret_cast<uint32_t*>(smem + L::vbuf_off);
    U* sk = reinterpret_cast<U*>(smem + L::sk_off);
    uint32_t* sv = reinterpret_cast<uint32_t*>(smem + L::sv_off);
    uint32_t* cnt = reinterpret_cast<uint32_t*>(smem + L::cnt_off);
    uint32_t* lb_cnt = reinterpret_cast<uint32_t*>(smem + L::lbc_off);  // LB_PAIR: each digit's tile count
    uint32_t* lb_start = lb_cnt + RADIX;                                // and tile-local start
    OFF* gbase = reinterpret_cast<OFF*>(smem + L::gbase_off);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + L::bar_off);
    int* misc = reinterpret_cast<int*>(smem + L::misc_off);  // [0..2] tile ids, [32..] warp totals

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t lt = lanemask_lt();
    PeerMasks<BITS> pm;
    pm.init(lane);
    const size_t portion_end = min(a.n, a.portion_begin + (size_t)a.portion_tiles * TILE);
    const bool bulk_ok = ((uintptr_t)src & 15) == 0 && (!PAIRS || first || ((uintptr_t)vsrc & 15) == 0);

    // The previous launch used the other look-back region; clear it for the next.
    {
        uint4* z = reinterpret_cast<uint4*>(a.lookback_next);
        const size_t nz = a.lookback_words / 4;
        for (size_t i = (size_t)blockIdx.x * THREADS + tid; i < nz; i += (size_t)gridDim.x * THREADS)
            z[i] = make_uint4(0u, 0u, 0u, 0u);
    }
    zero_counters<RANK_WARPS * RADIX, THREADS>(cnt, tid);
    if (tid == 0) {
        for (int b = 0; b < NBUF; ++b) mbar_init(&bars[b], 1);
        fence_mbar_init();
    }
    __syncthreads();

    // thread 0: start the copy of tile t into buffer b (full tiles from an
    // aligned source; anything else arrives without data and is loaded below)
    auto issue = [&](int t, int b) {
        const size_t base = a.portion_begin + (size_t)t * TILE;
        const bool full = base + TILE <= portion_end;
        if (full && bulk_ok) {
            fence_proxy_async_smem();
            const uint32_t bytes = TILE * sizeof(U) + ((PAIRS && !first) ? TILE * 4 : 0);
            mbar_arrive_expect_tx(&bars[b], bytes);
            bulk_g2s(kbuf + (size_t)b * TILE, src + base, TILE * sizeof(U), &bars[b]);
            if constexpr (PAIRS) {
                if (!first) bulk_g2s(vbuf + (size_t)b * TILE, vsrc + base, TILE * 4, &bars[b]);
            }
        } else {
            mbar_arrive_expect_tx(&bars[b], 0);
        }
    };

    uint32_t parity = 0;  // bit b: the phase buffer b's barrier completes next

    // The first live pass transforms keys as it loads them (and makes the
    // positions), the last undoes the transform as it writes. For float keys
    // and for pairs that is a compile-time choice (TAGGED: the tile body is
    // built for both); a signed key's transform is one XOR, done with a mask
    // that is the sign bit only in the first or last pass.
    // The digit of a key. With 8-bit digits it is one byte of the key: a
    // byte permute (one instruction) with a selector fixed for the launch
    // takes it out zero-extended, where a variable shift and a mask take two
    // (and a 64-bit shift more); 64-bit keys first pick the 32-bit half.
    const uint32_t byte_sel = 0x4440u | (uint32_t)((shift & 31) >> 3);
    auto dig = [&](U k) -> uint32_t {
        if constexpr (BITS == 8) {
            uint32_t w;
            if constexpr (sizeof(U) == 8) w = shift >= 32 ? (uint32_t)((uint64_t)k >> 32) : (uint32_t)k;
            else w = (uint32_t)k;
            return __byte_perm(w, 0u, byte_sel);
        } else {
            return digit_of(k, shift, MASK);
        }
    };

    constexpr bool TAGGED = XF == 2 || PAIRS;
    constexpr U SIGN = (U)((U)1 << (8 * sizeof(U) - 1));
    const U first_mask = (XF == 1 && first) ? SIGN : (U)0;
    const U last_mask = (XF == 1 && last) ? SIGN : (U)0;

    // One tile. FULL (a compile-time tag) drops every per-key bounds test:
    // only the last tile of a portion can be partial. FIRST is the
    // compile-time first-pass tag (false unless TAGGED).
    auto process = [&](int t, int b, auto full_tag, auto first_tag, auto unstable_tag) {
        constexpr bool FULL = decltype(full_tag)::value;
        constexpr bool FIRST = decltype(first_tag)::value;
        constexpr bool UNST = decltype(unstable_tag)::value;
        auto load_key = [&](U k) -> U {
            if constexpr (FIRST) return to_key<U, XF>(k);
            else if constexpr (XF == 1 && !TAGGED) return (U)(k ^ first_mask);
            else return k;
        };
        const size_t tile_base = a.portion_begin + (size_t)t * TILE;
        const int tile_n = FULL ? TILE : (int)min((size_t)TILE, portion_end - tile_base);
        U* kb = kbuf + (size_t)b * TILE;
        [[maybe_unused]] uint32_t* vb = vbuf + (size_t)b * TILE;

        // ---- 1. the tile's keys in shared memory
        if (!mbar_wait(&bars[b], (parity >> b) & 1u)) atomicOr(a.error, ERR_TIMEOUT);
        parity ^= 1u << b;
        if (!(FULL && bulk_ok)) {
            for (int i = tid; i < tile_n; i += THREADS) {
                kb[i] = src[tile_base + i];
                if constexpr (PAIRS) {
                    if (!first) vb[i] = vsrc[tile_base + i];
                }
            }
            __syncthreads();
        }

        // ---- 2. per-warp digit counts
        const int wbase = warp * 32 * IPT + lane;
        uint32_t* my_cnt = cnt + warp * RADIX;
        {
#pragma unroll
            for (int i = 0; i < IPT; ++i) {
                if (FULL || wbase + i * 32 < tile_n) {
                    const U k = load_key(kb[wbase + i * 32]);
                    atomicAdd(&my_cnt[dig(k)], 1u);
                }
            }
        }
        __syncthreads();

        // digit owners: prefix over warps, publish the tile's counts, tile-local starts
        // (an owner of DPT digits moves their counters as one 8- or 16-byte word)
        uint32_t tcount[DPT];
        uint32_t own = 0;
        if (tid < OWNERS) {
#pragma unroll
            for (int q = 0; q < DPT; ++q) tcount[q] = 0;
#pragma unroll
            for (int w = 0; w < RANK_WARPS; ++w) {
                uint32_t c[DPT];
                cnt_load<DPT>(cnt + w * RADIX + tid * DPT, c);
                cnt_store<DPT>(cnt + w * RADIX + tid * DPT, tcount);
#pragma unroll
                for (int q = 0; q < DPT; ++q) tcount[q] += c[q];
            }
#pragma unroll
            for (int q = 0; q < DPT; ++q) {
                own += tcount[q];
                if (t != 0 || !a.withhold_tile0)
                    st_relaxed_gpu(a.lookback + (size_t)t * RADIX + tid * DPT + q,
                                   (t == 0 ? LB_FLAG_INC : LB_FLAG_AGG) | tcount[q]);
            }
        }
        uint32_t x = own;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31 && warp < OWNER_WARPS) misc[32 + warp] = (int)x;
        __syncthreads();
        uint32_t lstart[DPT];
        if (tid < OWNERS) {
            uint32_t run = x - own;
            for (int w = 0; w < warp; ++w) run += (uint32_t)misc[32 + w];
#pragma unroll
            for (int q = 0; q < DPT; ++q) {
                const int r = tid * DPT + q;
                lstart[q] = run;
                if constexpr (LB_PAIR) {
                    lb_cnt[r] = tcount[q];
                    lb_start[r] = run;
                }
                run += tcount[q];
            }
#pragma unroll
            for (int w = 0; w < RANK_WARPS; ++w) {
                uint32_t c[DPT];
                cnt_load<DPT>(cnt + w * RADIX + tid * DPT, c);
#pragma unroll
                for (int q = 0; q < DPT; ++q) c[q] += lstart[q];
                cnt_store<DPT>(cnt + w * RADIX + tid * DPT, c);
            }
        }
        __syncthreads();

        if constexpr (UNST) {
            // ---- 3'. first pass of a keys-only sort: any order inside a digit
#pragma unroll
            for (int i = 0; i < IPT; ++i) {
                const int idx = wbase + i * 32;
                if (FULL || idx < tile_n) {
                    const U k = load_key(kb[idx]);
                    sk[atomicAdd(&my_cnt[dig(k)], 1u)] = k;
                }
            }
        } else if constexpr (RANK_AHEAD) {
            // ---- 3. as below, with the equals of item i + 1 found (ballots
            // and shuffles only, no memory) before item i's counter update,
            // so that the two overlap
            auto find = [&](int i, U& k, uint32_t& d, uint32_t& peers) {
                const int idx = wbase + i * 32;
                k = load_key(kb[FULL ? idx : min(idx, TILE - 1)]);
                d = dig(k);
                if ((i % MATCH_MOD) < MATCH_CNT) peers = __match_any_sync(0xffffffffu, d);
                else peers = pm.peers(d);
                if (!FULL) peers &= __ballot_sync(0xffffffffu, idx < tile_n);
            };
            U kn;
            uint32_t dn, pn;
            find(0, kn, dn, pn);
#pragma unroll
            for (int i = 0; i < IPT; ++i) {
                const int idx = wbase + i * 32;
                const U k = kn;
                const uint32_t d = dn, peers = pn;
                if (i + 1 < IPT) find(i + 1, kn, dn, pn);
                if (FULL || idx < tile_n) {
                    const uint32_t c = my_cnt[d];
                    my_cnt[d] = c + __popc(peers);
                    const uint32_t pos = c + __popc(peers & lt);
                    sk[pos] = k;
                    if constexpr (PAIRS) sv[pos] = FIRST ? (uint32_t)(tile_base + idx) : vb[idx];
                }
                __syncwarp();
            }
        } else {
            // ---- 3. rank among equal digits in the warp and stage in sorted order
#pragma unroll
            for (int i = 0; i < IPT; ++i) {
                const int idx = wbase + i * 32;
                const bool valid = FULL || idx < tile_n;
                const U k = load_key(kb[FULL ? idx : min(idx, TILE - 1)]);
                const uint32_t d = dig(k);
                uint32_t peers;
                if ((i % MATCH_MOD) < MATCH_CNT) peers = __match_any_sync(0xffffffffu, d);
                else peers = pm.peers(d);
                if (!FULL) peers &= __ballot_sync(0xffffffffu, valid);
                if (valid) {
                    const uint32_t c = my_cnt[d];
                    my_cnt[d] = c + __popc(peers);
                    const uint32_t pos = c + __popc(peers & lt);
                    sk[pos] = k;
                    if constexpr (PAIRS) sv[pos] = FIRST ? (uint32_t)(tile_base + idx) : vb[idx];
                }
                __syncwarp();
            }
        }

        // ---- 4. owners: keys of their digit in earlier tiles (the decoupled
        // look-back; predecessors have had the whole ranking pass to publish),
        // then the digit's global base
        if constexpr (LB_PAIR) {
            // two adjacent threads a digit: each loads LBW predecessors, the
            // pair covers 2 x LBW per round trip; the even thread publishes
            static_assert(2 * RADIX == THREADS && DPT == 1, "a pair of threads per digit");
            const int r = tid >> 1, h = tid & 1;
            const uint32_t pair = 3u << (lane & ~1);
            const uint32_t tc = lb_cnt[r];
            uint32_t excl = 0;
            if (t > 0) {
                int j = t - 1;
                uint32_t spins = 0;
                bool done = false;
                while (j >= 0 && !done) {
                    uint32_t w[LBW];
#pragma unroll
                    for (int k = 0; k < LBW; ++k) {
                        const int e = j - h * LBW - k;
                        w[k] = e >= 0 ? ld_relaxed_gpu(a.lookback + (size_t)e * RADIX + r) : LB_FLAG_INC;
                    }
                    int adv = 0;
                    uint32_t sum = 0;
                    bool stop = false, inc = false;
#pragma unroll
                    for (int k = 0; k < LBW; ++k) {
                        const uint32_t f = w[k] & ~LB_VALUE;
                        if (stop) continue;
                        if (f == 0) {
                            stop = true;
                            continue;
                        }
                        sum += w[k] & LB_VALUE;
                        ++adv;
                        if (f == LB_FLAG_INC) stop = inc = true;
                    }
                    // the older half counts only when the newer half was all aggregates
                    const int adv1 = __shfl_xor_sync(pair, adv, 1);
                    const uint32_t sum1 = __shfl_xor_sync(pair, sum, 1);
                    const int inc1 = __shfl_xor_sync(pair, (int)inc, 1);
                    const int adv0 = h ? adv1 : adv, adv_o = h ? adv : adv1;
                    const uint32_t sum0 = h ? sum1 : sum, sum_o = h ? sum : sum1;
                    const bool inc0 = h ? inc1 != 0 : inc, inc_o = h ? inc : inc1 != 0;
                    int step = adv0;
                    uint32_t add = sum0;
                    bool fin = inc0;
                    if (adv0 == LBW && !inc0) {
                        step += adv_o;
                        add += sum_o;
                        fin = inc_o;
                    }
                    excl += add;
                    j -= step;
                    done = fin;
                    if (step == 0 && ++spins > a.spin_limit) {
                        if (h == 0) atomicOr(a.error, ERR_TIMEOUT);
                        break;
                    }
                }
                if (h == 0) st_relaxed_gpu(a.lookback + (size_t)t * RADIX + r, LB_FLAG_INC | (excl + tc));
            }
            if (h == 0) {
                const unsigned long long carry = a.carry_in ? a.carry_in[r] : 0ull;
                unsigned long long start = bins[r] + carry + excl;
                if (start + tc > a.n) {  // only after a timeout: keep every write in bounds
                    atomicOr(a.error, ERR_BOUNDS);
                    start = a.n - tc;
                }
                gbase[r] = (OFF)((long long)start - (long long)lb_start[r]);
                if (a.carry_out && t == a.portion_tiles - 1) a.carry_out[r] = carry + excl + tc;
            }
        } else if (tid < OWNERS) {
#pragma unroll
            for (int q = 0; q < DPT; ++q) {
                const int r = tid * DPT + q;
                uint32_t excl = 0;
                if (t > 0) {
                    // LBW predecessors per round trip: their loads go out
                    // together, then they are summed newest first up to the
                    // first inclusive entry; an entry not yet published ends
                    // the round there and the next round starts from it
                    int j = t - 1;
                    uint32_t spins = 0;
                    bool done = false;
                    while (j >= 0 && !done) {
                        uint32_t w[LBW];
#pragma unroll
                        for (int k = 0; k < LBW; ++k)
                            w[k] = j - k >= 0 ? ld_relaxed_gpu(a.lookback + (size_t)(j - k) * RADIX + r) : LB_FLAG_INC;
                        int adv = 0;
                        bool stalled = false;
#pragma unroll
                        for (int k = 0; k < LBW; ++k) {
                            const uint32_t f = w[k] & ~LB_VALUE;
                            if (done || stalled) continue;
                            if (f == 0) {
                                stalled = true;
                                continue;
                            }
                            excl += w[k] & LB_VALUE;
                            ++adv;
                            if (f == LB_FLAG_INC) done = true;
                        }
                        j -= adv;
                        if (adv == 0 && ++spins > a.spin_limit) {
                            atomicOr(a.error, ERR_TIMEOUT);
                            break;
                        }
                    }
                    st_relaxed_gpu(a.lookback + (size_t)t * RADIX + r, LB_FLAG_INC | (excl + tcount[q]));
                }
                const unsigned long long carry = a.carry_in ? a.carry_in[r] : 0ull;
                unsigned long long start = bins[r] + carry + excl;
                if (start + tcount[q] > a.n) {  // only after a timeout: keep every write in bounds
                    atomicOr(a.error, ERR_BOUNDS);
                    start = a.n - tcount[q];
                }
                gbase[r] = (OFF)((long long)start - (long long)lstart[q]);
                if (a.carry_out && t == a.portion_tiles - 1) a.carry_out[r] = carry + excl + tcount[q];
            }
        }
        __syncthreads();
        if constexpr (NBUF == 1) {
            // every key of this tile sits in the staging tile now: the key
            // buffer takes the next tile's copy while this one is scattered
            if (tid == 0 && misc[1] < a.portion_tiles) issue(misc[1], 0);
        }

        // ---- 5. runs per digit to global memory (the last live pass undoes
        // the key transform as it writes)
        auto scatter = [&](auto last_tag) {
            constexpr bool LAST = decltype(last_tag)::value;
#pragma unroll
            for (int i = 0; i < SCATTER_IT; ++i) {
                const int s = i * THREADS + tid;
                if ((TILE % THREADS == 0 || i < SCATTER_IT - 1 || s < TILE) && (FULL || s < tile_n)) {
                    const U k = sk[s];
                    const OFF p = gbase[dig(k)] + (OFF)s;
                    if (write_keys) {
                        if constexpr (LAST) dst[p] = from_key<U, XF>(k);
                        else if constexpr (XF == 1) dst[p] = (U)(k ^ last_mask);
                        else dst[p] = k;
                    }
                    if constexpr (PAIRS) vdst[p] = sv[s];
                }
            }
        };
        if constexpr (XF == 2) {
            if (last) scatter(std::true_type{});
            else scatter(std::false_type{});
        } else {
            scatter(std::false_type{});
        }
        // clear the counters for the next tile (no one reads them past step 3)
        zero_counters<RANK_WARPS * RADIX, THREADS>(cnt, tid);
    };
    auto run_tile = [&](int t, int b) {
        const bool full = a.portion_begin + (size_t)(t + 1) * TILE <= portion_end;
        auto go = [&](auto first_tag, auto unstable_tag) {
            if (full) process(t, b, std::true_type{}, first_tag, unstable_tag);
            else process(t, b, std::false_type{}, first_tag, unstable_tag);
        };
        if constexpr (TAGGED) {
            if (first) {
                if constexpr (UNSTABLE1 && !PAIRS) go(std::true_type{}, std::true_type{});
                else go(std::true_type{}, std::false_type{});
            } else {
                go(std::false_type{}, std::false_type{});
            }
        } else if constexpr (UNSTABLE1 && !PAIRS) {
            if (first) go(std::false_type{}, std::true_type{});
            else go(std::false_type{}, std::false_type{});
        } else {
            go(std::false_type{}, std::false_type{});
        }
    };

    if constexpr (NBUF == 2) {
        if (tid == 0) {
            const int t0 = (int)atomicAdd(a.tile_counter, 1u);
            misc[0] = t0;
            if (t0 < a.portion_tiles) issue(t0, 0);
        }
        __syncthreads();
        int cur = misc[0], b = 0, it = 0;
        while (cur < a.portion_tiles) {
            if (tid == 0) {  // take the next tile and start its copy into the other buffer
                const int nx = (int)atomicAdd(a.tile_counter, 1u);
                misc[1 + (it & 1)] = nx;
                if (nx < a.portion_tiles) issue(nx, b ^ 1);
            }
            run_tile(cur, b);
            cur = misc[1 + (it & 1)];
            b ^= 1;
            ++it;
            __syncthreads();
        }
    } else {
        // one buffer: each CTA holds the claim on its next tile (misc[1])
        // while it works on this one (misc[0]) and brings that tile into L2;
        // once this tile's keys are ranked into the staging tile, the copy of
        // the next one into the key buffer starts (in process), so it runs
        // under this tile's look-back and scatter
        auto claim_next = [&]() {  // thread 0
            const int nx = (int)atomicAdd(a.tile_counter, 1u);
            misc[1] = nx;
            if (nx < a.portion_tiles) {
                const size_t nb = a.portion_begin + (size_t)nx * TILE;
                const size_t ne = min(portion_end, nb + TILE);
                prefetch_l2(src + nb, src + ne);
                if constexpr (PAIRS) {
                    if (!first) prefetch_l2(vsrc + nb, vsrc + ne);
                }
            }
        };
        if (tid == 0) {
            const int t = (int)atomicAdd(a.tile_counter, 1u);
            misc[0] = t;
            if (t < a.portion_tiles) {
                issue(t, 0);
                claim_next();
            }
        }
        __syncthreads();
        for (;;) {
            const int t = misc[0];
            if (t >= a.portion_tiles) break;
            run_tile(t, 0);
            __syncthreads();
            if (tid == 0) {
                const int t2 = misc[1];  // its copy was issued by run_tile
                misc[0] = t2;
                if (t2 < a.portion_tiles) claim_next();
            }
            __syncthreads();
        }
    }
}

}  // namespace ts
