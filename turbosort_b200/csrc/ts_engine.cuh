// ts_engine.cuh — host-side drivers that enqueue one device sort.
//
// The tier choice follows the crate's dispatcher (src/dispatch.rs:31-111):
// n <= 1 is a no-op; one-byte keys take the counting sort
// (src/radix/mod.rs:123-164); short slices take the on-chip tiers
// (src/tiny.rs, src/small.rs: one warp's register bitonic network up to 256
// keys, and up to 1024 keys of 4 bytes or 512 of 8; then one CTA, by the MSD
// routine for 4- and 8-byte keys and a shared-memory bitonic network for
// 1- and 2-byte keys, up to 4096); the rest runs the LSD
// passes (src/radix/mod.rs:180-271). The presorted early-out
// (src/presorted.rs:15-65) and the constant-digit skip are decided on the
// device, so nothing in a sort waits on the host.
#pragma once

#include <algorithm>
#include <cstring>
#include <type_traits>

#include "ts_coop.cuh"
#include "ts_ctx.h"
#include "ts_divert.cuh"
#include "ts_lsd.cuh"
#include "ts_onesweep.cuh"
#include "ts_small.cuh"

namespace ts {

// Tile shapes per key width; 8-bit digits. A tile is 16 warps x 32 lanes x
// IPT keys. Variant V halves the keys a thread V times: smaller tiles give a
// short sort more CTAs to run on (2^20 u32 keys fill only 93 of the largest
// tiles), larger ones cost less per key on long sorts; the autotuner
// (ts_lsd_autotune) picks a variant per key width and length bin.
constexpr int LSD_VARIANTS = 3;
constexpr int LSD_BINS = 3;  // n < 2^22, n < 2^25, larger
static inline int lsd_bin(size_t n) { return n < ((size_t)1 << 22) ? 0 : n < ((size_t)1 << 25) ? 1 : 2; }

// Digit widths of the plain LSD: 8 bits by default (the crate's byte core,
// src/radix/mod.rs:205-271); keys-only sorts below 2^31 keys can also run
// 4..11-bit digits (the crate's wide core takes 11, src/radix/mod.rs:43-54,
// 518-600), chosen per key width and length bin (ts_lsd_digit_bits, or the
// autotuner).
constexpr int LSD_MIN_BITS = 4;
constexpr int LSD_MAX_BITS = 11;

template <typename U, bool PAIRS, int V = 0, int B = 8>
struct LsdCfg {
    static constexpr int BITS = B;
    static_assert(B >= LSD_MIN_BITS && B <= LSD_MAX_BITS && (B == 8 || (!PAIRS && V == 0)), "digit width");
    static constexpr int THREADS = 512;
    // the first live pass of a keys-only sort ranks with shared atomics
    // (k_onesweep, UNSTABLE1)
    static constexpr bool UNSTABLE1 = true;
    // the next item's equals found before this item's counter update
    // (k_onesweep; 2^28 u32 4.26 -> 4.21 ms, 2^27 u64 without diverting
    // 6.69 -> 6.60 ms)
    static constexpr bool RANK_AHEAD = true;
    // look-back entries loaded per round trip
    static constexpr int LBW = LB_WINDOW;
    // two threads walk each digit's look-back (k_onesweep LB_PAIR): 2^27 u64
    // keys without diverting 6.62 -> 6.47 ms; 2^28 u32 keys 4.22 -> 4.38 ms,
    // so 8-byte keys only
    static constexpr bool LB_PAIR = sizeof(U) == 8 && !PAIRS && B == 8;
    // 8-byte keys without positions divert (src/radix/divert.rs): the plan may
    // leave out the lowest live digits, and k_divert_runs / k_divert_long
    // finish the runs that leaves
    static constexpr bool DIVERT = !PAIRS && sizeof(U) == 8 && B == 8;
    // 64-bit offsets (more than 2^31 keys) are compiled for 8-bit digits only
    static constexpr bool HUGE_OK = B == 8;
    // the largest tile for which two CTAs (one tile of keys and positions, the
    // staging tile, 32-bit per-warp counters) share one SM's shared memory:
    // the per-tile costs (look-back, counter scans) shrink per key as tiles
    // grow, which on a B200 outweighs double-buffering a smaller tile
    // (2^28 u32 keys: 15 keys a thread double-buffered 5.18 ms, 22 single 4.83 ms)
    static constexpr int IPT0 = sizeof(U) == 8 ? (PAIRS ? 7 : 11) : (PAIRS ? 11 : (sizeof(U) == 4 ? 22 : 32));
    // Other digit widths (keys only): per-warp counters take 16 x 2^B words,
    // so wider digits leave less room for the tile. The largest tile (up to
    // IPT0 keys a thread) with which two CTAs still share an SM, if that
    // leaves at least 8 keys a thread; else the largest for one CTA an SM.
    static constexpr int fit_ipt(size_t budget) {
        const size_t fixed = (size_t)16 * (1u << B) * 4 + (size_t)(1u << B) * 8 + 1024;
        return budget > fixed ? (int)((budget - fixed) / (2 * sizeof(U) * THREADS)) : 0;
    }
    static constexpr int ipt_for_bits() {
        return fit_ipt(113 * 1024) >= 8 ? (fit_ipt(113 * 1024) < IPT0 ? fit_ipt(113 * 1024) : IPT0)
                                        : (fit_ipt(226 * 1024) < IPT0 ? fit_ipt(226 * 1024) : IPT0);
    }
    static constexpr int IPT = B == 8 ? IPT0 >> V : ipt_for_bits();
    static_assert(V >= 0 && V < LSD_VARIANTS && IPT >= 1, "tile variant");
    static constexpr int NBUF = 1;  // tiles of keys in flight per CTA; the next one is prefetched into L2
    // items with i % MATCH_MOD < MATCH_CNT find their digit's peers with
    // match.any, the rest with ballots: a share of the items keeps the match
    // unit busy without making it the bottleneck and takes that share of the
    // ranking off the integer pipe (2^28 u32 keys on a B200, one in four:
    // 5.81 -> 5.19 ms a sort; with the unstable first pass, u32 one in three
    // 4.32 ms, one in four 4.34, one in five 4.41; u64 one in four 6.58, one
    // in three 6.71)
    static constexpr int MATCH_MOD = (sizeof(U) == 8 || PAIRS) ? 4 : 3;
    static constexpr int MATCH_CNT = 1;
    using Smem = SweepSmem<U, BITS, THREADS, IPT, PAIRS, NBUF, LB_PAIR>;
    static_assert(Smem::bytes <= 227 * 1024, "one CTA's shared memory");
    static constexpr int TILE = Smem::TILE;
    static constexpr int RADIX = 1 << BITS;
    static constexpr int ND = (Bits<U>::W + BITS - 1) / BITS;
};

// Layout of ctx->meta for one sort.
struct MetaLayout {
    size_t scan_off, plan_off, counters_off, hist_off, bins_off, carry_off, bytes;
    static MetaLayout make(int nd, int radix, int launches) {
        MetaLayout m{};
        size_t o = 0;
        m.scan_off = o;
        o += 256;
        m.plan_off = o;
        o += 512;
        m.counters_off = o;
        o += ((size_t)launches * 4 + 255) / 256 * 256;
        m.hist_off = o;
        o += (size_t)nd * radix * 8;
        m.bins_off = o;
        o += (size_t)nd * radix * 8;
        m.carry_off = o;
        o += (size_t)2 * radix * 8;
        m.bytes = o;
        return m;
    }
    size_t zero_bytes() const { return bins_off; }  // scan state .. histograms
    // in the (zeroed) plan area, after the Plan: the diverted sort's count of
    // listed runs (u64) and its work counter (u32)
    size_t divert_off() const { return plan_off + 128; }
    // after those: the largest bucket of each digit (u64, 0 when not live),
    // which the plan writes
    size_t maxb_off() const { return plan_off + 144; }
};
static_assert(sizeof(Plan) <= 128, "the plan area holds the Plan and the divert counters");

// Resident CTAs per SM for `kernel`, raising its dynamic shared memory limit
// first when it needs more than the default 48 KB. Cached per kernel.
int occupancy_of(const void* kernel, int threads, size_t smem);
template <typename K>
static int occupancy(ts_ctx*, K kernel, int threads, size_t smem) {
    return occupancy_of((const void*)kernel, threads, smem);
}

static inline bool aligned16(const void* p) { return ((uintptr_t)p & 15) == 0; }

// A launch on the context's stream that may begin while the previous kernel
// in the stream finishes (programmatic stream serialization): the kernel
// calls dep_wait() before it reads or writes anything, so only the launch
// latency overlaps.
template <typename... KArgs, typename... Args>
static cudaError_t launch_dep(ts_ctx* c, void (*kernel)(KArgs...), int grid, int block, size_t smem, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = c->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}
// row of the per-width tuning tables: 1, 2, 4, 8 bytes
static inline int width_slot(size_t bytes) { return bytes == 1 ? 0 : bytes == 2 ? 1 : bytes == 4 ? 2 : 3; }

// The LSD passes over `in` (n keys), writing through pp[0]/pp[1]; with PAIRS
// the positions ping-pong through vpp and the last pass writes `vout`.
template <typename U, int XF, bool PAIRS, typename C = LsdCfg<U, PAIRS>>
static ts_status run_lsd(ts_ctx* c, const U* in, U* pp0, U* pp1, uint32_t* vpp0, uint32_t* vpp1, uint32_t* vout,
                         size_t n, int write_keys_last, Plan** plan_out) {
    constexpr int RADIX = C::RADIX, ND = C::ND, TILE = C::TILE;
    const size_t tiles = (n + TILE - 1) / TILE;
    const size_t max_portion_tiles = (size_t)(LB_VALUE / TILE);
    const int portions = (int)((tiles + max_portion_tiles - 1) / max_portion_tiles);
    const size_t portion_tiles = std::min(tiles, max_portion_tiles);
    const int launches = ND * portions;
    const MetaLayout m = MetaLayout::make(ND, RADIX, launches);
    ts_status s;
    if ((s = grow(c, c->meta, m.bytes, "sort metadata")) != TS_OK) return s;
    const size_t lb_words = portion_tiles * RADIX;
    if ((s = grow(c, c->lookback, 2 * lb_words * 4, "look-back")) != TS_OK) return s;
    char* meta = (char*)c->meta.p;
    ScanState* st = (ScanState*)(meta + m.scan_off);
    Plan* plan = (Plan*)(meta + m.plan_off);
    uint32_t* counters = (uint32_t*)(meta + m.counters_off);
    unsigned long long* hist = (unsigned long long*)(meta + m.hist_off);
    unsigned long long* bins = (unsigned long long*)(meta + m.bins_off);
    unsigned long long* carry = (unsigned long long*)(meta + m.carry_off);
    uint32_t* lb = (uint32_t*)c->lookback.p;
    const int vec_ok = aligned16(in);

    mark(c, "scan");
    TS_CUDA(c, cudaMemsetAsync(meta, 0, m.zero_bytes(), c->stream));
    {
        constexpr int T = 256;
        const int grid = c->sm_count * 4;
        k_scan<U, XF, T><<<grid, T, 0, c->stream>>>(in, n, C::BITS, ND, st, vec_ok, (uint4*)lb, lb_words / 4);
        ++c->launches;
    }
    mark(c, "histogram");
    {
        constexpr int T = 1024;
        const size_t smem = (size_t)ND * RADIX * hist_copies<RADIX, ND>() * 4;
        static_assert(144 + 8 * ND <= 512, "the plan area holds every digit's largest bucket");
        auto kern = k_hist<U, XF, C::BITS, T, C::DIVERT>;
        const int occ = occupancy(c, kern, T, smem);
        TS_CUDA(c, launch_dep(c, kern, c->sm_count * occ, T, smem, in, n, st, hist, vec_ok, bins, plan, PAIRS ? 1 : 0,
                              (unsigned long long*)(meta + m.maxb_off()), c->divert ? 1 : 0));
        ++c->launches;
    }
    {
        using Sm = typename C::Smem;
        auto kern = k_onesweep<U, XF, C::BITS, C::THREADS, C::IPT, PAIRS, C::NBUF, false, C::MATCH_MOD, C::MATCH_CNT,
                               C::UNSTABLE1, C::RANK_AHEAD, C::LBW, C::LB_PAIR>;
        if constexpr (C::HUGE_OK) {
            if (n > (size_t)0x7fffffff)
                kern = k_onesweep<U, XF, C::BITS, C::THREADS, C::IPT, PAIRS, C::NBUF, true, C::MATCH_MOD, C::MATCH_CNT,
                                  C::UNSTABLE1, C::RANK_AHEAD, C::LBW, C::LB_PAIR>;
        } else {
            if (n > (size_t)0x7fffffff) return fail(c, TS_ERR_INTERNAL, "digit width without 64-bit offsets");
        }
        const int occ = occupancy(c, kern, C::THREADS, Sm::bytes);
        SweepArgs<U, PAIRS> a{};
        a.in = in;
        a.pp[0] = pp0;
        a.pp[1] = pp1;
        a.vpp[0] = vpp0;
        a.vpp[1] = vpp1;
        a.vout = vout;
        a.n = n;
        a.write_keys_last = write_keys_last;
        a.plan = plan;
        a.bins = bins;
        a.error = c->d_error;
        a.spin_limit = c->test_spin_limit ? c->test_spin_limit : SPIN_LIMIT;
        int launch = 0;
        for (int slot = 0; slot < ND; ++slot) {
            for (int q = 0; q < portions; ++q, ++launch) {
                a.slot = slot;
                a.portion_begin = (size_t)q * portion_tiles * TILE;
                a.portion_tiles = (int)std::min(portion_tiles, tiles - (size_t)q * portion_tiles);
                a.carry_in = portions > 1 && q > 0 ? carry + (size_t)(q & 1) * RADIX : nullptr;
                a.carry_out = portions > 1 ? carry + (size_t)((q + 1) & 1) * RADIX : nullptr;
                a.lookback = lb + (size_t)(launch & 1) * lb_words;
                a.lookback_next = lb + (size_t)((launch + 1) & 1) * lb_words;
                a.lookback_words = lb_words;
                a.tile_counter = counters + launch;
                a.withhold_tile0 = c->test_spin_limit != 0 && launch == 0;
                const int grid = (int)std::min((size_t)c->sm_count * occ, (size_t)a.portion_tiles);
                mark(c, "onesweep");
                TS_CUDA(c, launch_dep(c, kern, grid, C::THREADS, Sm::bytes, a));
                ++c->launches;
            }
        }
    }
    c->test_spin_limit = 0;  // the test hook covers one sort
    *plan_out = plan;
    return TS_OK;
}

// The whole LSD of a keys-only sort of 2- or 4-byte keys in one cooperative
// launch (k_lsd_coop), with tiles of IPT keys a thread; false in *ran when the
// slice has more tiles than CTAs that can be resident at once.
template <typename U, int XF, int IPT>
static ts_status run_lsd_coop_ipt(ts_ctx* c, U* d_data, U* d_alt, size_t n, bool* ran) {
    using L = CoopSmem<U, IPT>;
    constexpr int ND = (int)sizeof(U);
    auto kern = k_lsd_coop<U, XF, IPT>;
    const int occ = std::min(2, occupancy_of((const void*)kern, COOP_THREADS, L::bytes));
    const size_t tiles = (n + L::TILE - 1) / L::TILE;
    *ran = false;
    if (tiles > (size_t)occ * c->sm_count || tiles > (size_t)COOP_THREADS) return TS_OK;
    // meta: the Plan where every LSD keeps it, the barrier state, the digit
    // counts and the tile counts (zeroed: no pass's tag)
    const MetaLayout ml = MetaLayout::make(1, 1, 0);
    const size_t state_off = 1024;  // after the plan area
    static_assert(sizeof(Plan) + 256 <= 1024, "the plan area ends before the barrier state");
    const size_t hist_off = (state_off + sizeof(CoopState) + 255) / 256 * 256;
    const size_t tcnt_off = hist_off + (size_t)ND * 256 * 4;
    const size_t end = tcnt_off + tiles * 256 * 2;
    ts_status s;
    if ((s = grow(c, c->meta, end, "sort metadata")) != TS_OK) return s;
    char* meta = (char*)c->meta.p;
    mark(c, "single-launch LSD");
    TS_CUDA(c, cudaMemsetAsync(meta, 0, end, c->stream));
    CoopArgs<U> a{};
    a.data = d_data;
    a.alt = d_alt;
    a.n = n;
    a.st = (CoopState*)(meta + state_off);
    a.hist = (unsigned int*)(meta + hist_off);
    a.tcnt = (unsigned short*)(meta + tcnt_off);
    a.plan = (Plan*)(meta + ml.plan_off);
    a.maxb = (unsigned long long*)(meta + ml.maxb_off());
    a.error = c->d_error;
    a.spin_limit = c->test_spin_limit ? c->test_spin_limit : SPIN_LIMIT;
    a.withhold_cta0 = c->test_spin_limit != 0;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)tiles);
    cfg.blockDim = dim3(COOP_THREADS);
    cfg.dynamicSmemBytes = L::bytes;
    cfg.stream = c->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    TS_CUDA(c, cudaLaunchKernelEx(&cfg, kern, a));
    ++c->launches;
    c->test_spin_limit = 0;
    *ran = true;
    return TS_OK;
}

// The smallest tile that fits the slice into one wave gives the most CTAs.
// Tiles of 22 keys a thread (one wave of up to 3.3M keys) were slower than
// the multi-launch sort from 2M keys on (a B200: 0.125 against 0.110 ms at
// 2^21, whose 187 tiles give 39 SMs two), so the largest tile is 11 keys a
// thread (1,667,072 keys on 148 SMs).
constexpr int COOP_MAX_IPT = 11;
template <typename U, int XF>
static ts_status run_lsd_coop(ts_ctx* c, U* d_data, U* d_alt, size_t n, bool* ran) {
    ts_status s = run_lsd_coop_ipt<U, XF, 7>(c, d_data, d_alt, n, ran);
    if (s != TS_OK || *ran) return s;
    return run_lsd_coop_ipt<U, XF, COOP_MAX_IPT>(c, d_data, d_alt, n, ran);
}
// keys a single-launch sort can take on this GPU (one wave of its largest tiles)
template <typename U, int XF>
static size_t coop_capacity(ts_ctx* c) {
    using L = CoopSmem<U, COOP_MAX_IPT>;
    const int occ = std::min(2, occupancy_of((const void*)k_lsd_coop<U, XF, COOP_MAX_IPT>, COOP_THREADS, L::bytes));
    return std::min((size_t)occ * c->sm_count, (size_t)COOP_THREADS) * L::TILE;
}

// The LSD passes of a keys-only sort of n <= 2^31 - 1 keys at a digit width
// of LSD_MIN_BITS..LSD_MAX_BITS other than 8 (sorted keys end in d_data or,
// after an odd pass count, d_alt, as the plan says). Compiled apart from the
// 8-bit sorts, in ts_width_*.cu.
template <typename U, int XF>
ts_status run_lsd_bits(ts_ctx* c, int bits, U* d_data, U* d_alt, size_t n, Plan** plan);

template <typename U, int XF>
ts_status sort_keys_device(ts_ctx* c, U* d_data, size_t n, U* d_alt) {
    if (n <= 1) return TS_OK;
    if constexpr (sizeof(U) == 1) {
        if (n > (size_t)SMALL_MAX) {
            ts_status s;
            if ((s = grow(c, c->meta, 256 * 8, "counts")) != TS_OK) return s;
            unsigned long long* h = (unsigned long long*)c->meta.p;
            mark(c, "count8");
            TS_CUDA(c, cudaMemsetAsync(h, 0, 256 * 8, c->stream));
            k_count8<XF><<<c->sm_count * 4, 512, 0, c->stream>>>((const uint8_t*)d_data, n, h);
        ++c->launches;
            mark(c, "fill8");
            const size_t work = (n + 15) / 16;
            const int grid = (int)std::min((work + 255) / 256, (size_t)c->sm_count * 8);
            k_fill8<XF><<<grid, 256, 0, c->stream>>>((uint8_t*)d_data, n, h);
            ++c->launches;
            mark(c, "end");
            c->last_tier = 2;
            return TS_OK;
        }
    }
    if (n <= (size_t)SMALL_MAX) {
        mark(c, "small");
        if (n <= 32) {
            k_warp_sort<U, XF, 1><<<1, 32, 0, c->stream>>>(d_data, (int)n);
        } else if (n <= (size_t)WARP_TIER_MAX) {
            k_warp_sort<U, XF, WARP_TIER_MAX / 32><<<1, 32, 0, c->stream>>>(d_data, (int)n);
        } else if (n <= 512 && sizeof(U) == 8) {
            k_warp_sort<U, XF, 16><<<1, 32, 0, c->stream>>>(d_data, (int)n);
        } else if (n <= 1024 && sizeof(U) <= 4) {
            k_warp_sort<U, XF, 32><<<1, 32, 0, c->stream>>>(d_data, (int)n);
        } else if constexpr (sizeof(U) >= 4) {
            // the one-CTA MSD routine; its CTA-level LSD fallback (keys crowding
            // one sub-range) needs a second buffer of n keys
            ts_status s;
            if (!d_alt) {
                if ((s = grow(c, c->alt, n * sizeof(U), "scratch keys")) != TS_OK) return s;
                d_alt = (U*)c->alt.p;
            }
            occupancy_of((const void*)k_msd_slice<U, XF>, SEG_THREADS, MSD_SMEM);
            k_msd_slice<U, XF><<<1, SEG_THREADS, MSD_SMEM, c->stream>>>(d_data, d_alt, (int)n);
        } else {
            const int threads = (int)std::min<size_t>(SMALL_THREADS, std::max<size_t>(32, (n + 1) / 2));
            k_small_sort<U, XF, false><<<1, threads, 0, c->stream>>>(d_data, d_data, nullptr, (int)n, 1);
        }
        ++c->launches;
        mark(c, "end");
        c->last_tier = 1;
        return TS_OK;
    }
    if constexpr (sizeof(U) > 1) {
        c->last_tier = 3;
        ts_status s;
        if (!d_alt) {
            if ((s = grow(c, c->alt, n * sizeof(U), "scratch keys")) != TS_OK) return s;
            d_alt = (U*)c->alt.p;
        }
        constexpr bool DIVERT = LsdCfg<U, false>::DIVERT;
        // a diverted sort lists the starts of its runs longer than DIVERT_SHORT
        const size_t runs_cap = n / (DIVERT_SHORT + 1) + 1;
        if constexpr (DIVERT) {
            if ((s = grow(c, c->runs, runs_cap * 8, "divert runs")) != TS_OK) return s;
            occupancy_of((const void*)k_divert_long<U, XF>, SEG_THREADS, MSD_SMEM);
        }
        const int variant = c->lsd_variant[width_slot(sizeof(U))][lsd_bin(n)];
        // a digit width other than 8 (keys below 2^31 only); it never diverts
        const int bits = n <= (size_t)0x7fffffff ? c->lsd_bits[width_slot(sizeof(U))][lsd_bin(n)] : 8;
        c->last_bits = bits;
        // 2- and 4-byte keys that fit one wave of tiles: the whole sort in one launch
        bool coop = false;
        if constexpr (sizeof(U) == 2 || sizeof(U) == 4) coop = bits == 8 && c->coop && n <= coop_capacity<U, XF>(c);
        c->last_tier = coop ? 4 : 3;
        auto enqueue = [&]() -> ts_status {
            Plan* plan = nullptr;
            ts_status st;
            if constexpr (sizeof(U) == 2 || sizeof(U) == 4) {
                if (coop) {
                    bool ran = false;
                    if ((st = run_lsd_coop<U, XF>(c, d_data, d_alt, n, &ran)) != TS_OK) return st;
                    if (!ran) return fail(c, TS_ERR_INTERNAL, "single-launch sort: more tiles than one wave");
                    mark(c, "end");
                    return TS_OK;
                }
            }
            if (bits != 8)
                st = run_lsd_bits<U, XF>(c, bits, d_data, d_alt, n, &plan);
            else if (variant == 1)
                st = run_lsd<U, XF, false, LsdCfg<U, false, 1>>(c, d_data, d_alt, d_data, nullptr, nullptr, nullptr, n,
                                                                1, &plan);
            else if (variant == 2)
                st = run_lsd<U, XF, false, LsdCfg<U, false, 2>>(c, d_data, d_alt, d_data, nullptr, nullptr, nullptr, n,
                                                                1, &plan);
            else
                st = run_lsd<U, XF, false>(c, d_data, d_alt, d_data, nullptr, nullptr, nullptr, n, 1, &plan);
            if (st != TS_OK) return st;
            mark(c, "finish");
            const int grid = c->sm_count * 4;
            TS_CUDA(c, launch_dep(c, k_finish_keys<U>, grid, 512, 0, (const Plan*)plan, (const U*)d_alt, d_data, n,
                                  (int)(aligned16(d_alt) && aligned16(d_data))));
            ++c->launches;
            if constexpr (DIVERT) {
                if (bits == 8) {
                    const MetaLayout m = MetaLayout::make(LsdCfg<U, false>::ND, LsdCfg<U, false>::RADIX, 0);
                    char* dv = (char*)c->meta.p + m.divert_off();
                    unsigned long long* n_runs = (unsigned long long*)dv;
                    unsigned int* counter = (unsigned int*)(dv + 8);
                    mark(c, "divert");
                    k_divert_runs<U, XF><<<c->sm_count * 8, 256, 0, c->stream>>>(
                        plan, d_data, n, (unsigned long long*)c->runs.p, n_runs, runs_cap, c->d_error, aligned16(d_data));
                    k_divert_long<U, XF><<<c->sm_count, SEG_THREADS, MSD_SMEM, c->stream>>>(
                        plan, d_data, d_alt, n, (const unsigned long long*)c->runs.p, n_runs, counter, c->d_error);
                    c->launches += 2;
                }
            }
            mark(c, "end");
            return TS_OK;
        };
        // Repeated calls with the same pointers and size replay the launch
        // sequence as a CUDA graph (no per-launch host cost): captured on the
        // second identical call, when every buffer already has its size. Not
        // while per-kernel timing is on, nor inside the caller's own capture.
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (c->stream) cudaStreamIsCapturing(c->stream, &cs);
        if (!c->use_graphs || !c->stream || c->timing || c->test_spin_limit || cs != cudaStreamCaptureStatusNone)
            return enqueue();
        const size_t key[9] = {sizeof(U) | (size_t)XF << 4 | (size_t)variant << 8 | (size_t)(c->divert ? 1 : 0) << 12 |
                                   (size_t)bits << 16 | (size_t)(coop ? 1 : 0) << 24,
                               (size_t)d_data, (size_t)d_alt, n,
                               (size_t)c->meta.p, (size_t)c->lookback.p, (size_t)c->d_error, (size_t)c->alt.p,
                               (size_t)c->runs.p};
        if (c->sort_graph && std::memcmp(key, c->sort_graph_key, sizeof key) == 0) {
            TS_CUDA(c, cudaGraphLaunch(c->sort_graph, c->stream));
            c->launches += c->sort_graph_launches;
            return TS_OK;
        }
        if (std::memcmp(key, c->sort_last_key, sizeof key) != 0) {
            std::memcpy(c->sort_last_key, key, sizeof key);
            return enqueue();
        }
        if (c->sort_graph) {
            cudaGraphExecDestroy(c->sort_graph);
            c->sort_graph = nullptr;
        }
        const unsigned long long before = c->launches;
        TS_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        c->capturing = true;
        s = enqueue();
        c->capturing = false;
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(c->stream, &g);
        if (s != TS_OK) {
            if (g) cudaGraphDestroy(g);
            return s;
        }
        if (e != cudaSuccess) return cuda_fail(c, e, "cudaStreamEndCapture");
        e = cudaGraphInstantiate(&c->sort_graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            c->sort_graph = nullptr;
            return cuda_fail(c, e, "cudaGraphInstantiate");
        }
        std::memcpy(c->sort_graph_key, key, sizeof key);
        c->sort_graph_launches = c->launches - before;
        TS_CUDA(c, cudaGraphLaunch(c->sort_graph, c->stream));
        return TS_OK;
    }
    return TS_OK;
}

template <typename U, int XF>
ts_status order_device(ts_ctx* c, const U* d_keys, size_t n, uint32_t* d_order) {
    if (n == 0) return TS_OK;
    if (n > 0xffffffffull) return fail(c, TS_ERR_TOO_LARGE, "sort_by_key: more than u32::MAX elements");
    if (n <= (size_t)SMALL_MAX) {
        mark(c, "small");
        const int threads = (int)std::min<size_t>(SMALL_THREADS, std::max<size_t>(32, (n + 1) / 2));
        k_small_sort<U, XF, true><<<1, threads, 0, c->stream>>>(d_keys, nullptr, d_order, (int)n, 0);
        ++c->launches;
        mark(c, "end");
        return TS_OK;
    }
    ts_status s;
    if ((s = grow(c, c->alt, 2 * n * sizeof(U) + 16, "scratch keys")) != TS_OK) return s;
    if ((s = grow(c, c->vals0, n * 4, "positions")) != TS_OK) return s;
    if ((s = grow(c, c->vals1, n * 4, "positions")) != TS_OK) return s;
    U* k0 = (U*)c->alt.p;
    U* k1 = (U*)((char*)c->alt.p + (n * sizeof(U) + 15) / 16 * 16);
    Plan* plan = nullptr;
    if ((s = run_lsd<U, XF, true>(c, d_keys, k0, k1, (uint32_t*)c->vals0.p, (uint32_t*)c->vals1.p, d_order, n, 0,
                                  &plan)) != TS_OK)
        return s;
    mark(c, "finish");
    k_iota_if_unsorted<<<c->sm_count * 4, 512, 0, c->stream>>>(plan, d_order, n);
        ++c->launches;
    mark(c, "end");
    return TS_OK;
}

}  // namespace ts
