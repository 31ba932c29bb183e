// ts_coop.cuh — the whole LSD sort of a short slice in one cooperative launch.
//
// The crate's LSD (src/radix/mod.rs:180-271): varying bits and sortedness
// (src/radix/histogram.rs:55-68, src/presorted.rs:15-65), every digit's
// histogram in one read (src/radix/histogram.rs:15-110), live passes
// (src/radix/mod.rs:229-239), one stable scatter per live digit
// (src/radix/scatter.rs:26-247) and the copy back after an odd pass count.
//
// A multi-launch sort of 2^20 keys is bound by latency, not bandwidth: four
// kernels before the first pass, a launch per pass, and in each pass a
// decoupled look-back whose inclusive prefixes travel a few tiles per L2
// round trip. Here every tile of the slice belongs to one resident CTA of a
// single cooperative launch (at most two CTAs an SM):
//   0. each CTA loads its tile as radix keys, ORs key ^ first key, checks the
//      order of adjacent keys (including the one before its tile) and counts
//      every digit; the totals go to global memory; grid barrier;
//      every CTA derives the same plan (mode, live digits) and every digit's
//      start in its histogram;
//   per live digit:
//   1. (after a grid barrier, from the second pass on) the CTA loads its
//      tile of the previous pass's output;
//   2. per-warp digit counts; the tile's counts are published at once, each
//      16-bit field tagged with the pass; tile-local starts; the keys ranked
//      into a staging tile (stable: warp, item, lane);
//   3. the CTA sums the published counts of every earlier tile (re-reading
//      a word until all of its fields carry this pass's tag): the keys of
//      each digit that come before this tile's;
//   4. each digit's global start = its start in the histogram plus that sum;
//      the staging tile goes out as runs per digit.
// Every wait is bounded: a grid barrier or a tag wait that runs out sets
// ERR_TIMEOUT and an abort word that ends every other wait, and the kernel
// returns.
#pragma once

#include <type_traits>

#include "ts_common.cuh"
#include "ts_onesweep.cuh"

namespace ts {

// Grid barrier arrivals go to COOP_CTRS counters (CTA t to counter t mod
// COOP_CTRS), each on its own 128-byte line, so that a few hundred arrivals do
// not queue on one address; one warp polls all of them at once.
constexpr int COOP_CTRS = 16;
constexpr int COOP_CTR_STRIDE = 32;  // words

struct CoopState {
    unsigned int arrive[COOP_CTRS * COOP_CTR_STRIDE];  // monotonic within a launch
    unsigned int abort;       // set when a wait ran out: every later wait returns at once
    unsigned int flags;       // SCAN_NOT_ASC | SCAN_NOT_DESC
    unsigned long long diff;  // OR of (radix key ^ first radix key)
};

template <typename U>
struct CoopArgs {
    U* data;              // keys, sorted in place
    U* alt;               // scratch of n keys
    size_t n;
    CoopState* st;        // zeroed before the launch
    unsigned int* hist;   // [ND][256] digit counts, zeroed before the launch
    unsigned short* tcnt; // [tiles][256] tile counts: (pass + 1) << 13 | count, zeroed before the launch
    Plan* plan;           // written by CTA 0, for ts_ctx_last_sort_info
    unsigned long long* maxb;  // [ND] each live digit's largest bucket (0: not live), written by CTA 0
    uint32_t* error;
    uint32_t spin_limit;  // barrier rounds without progress before ERR_TIMEOUT
    int withhold_cta0;    // test hook: CTA 0 never arrives at the first barrier
};

constexpr int COOP_THREADS = 512;
constexpr int COOP_WARPS = COOP_THREADS / 32;
// a published tile count: 13 bits of count under a 3-bit pass tag
constexpr int COOP_COUNT_BITS = 13;
constexpr uint32_t COOP_COUNT_MASK = (1u << COOP_COUNT_BITS) - 1;

// all eight 16-bit fields of w carry `tag`
__device__ __forceinline__ bool coop_tagged(const uint4& w, unsigned int tag) {
    const uint32_t t2 = tag << COOP_COUNT_BITS | tag << (16 + COOP_COUNT_BITS);
    const uint32_t m = ~(COOP_COUNT_MASK | COOP_COUNT_MASK << 16);
    return ((w.x & m) == t2) & ((w.y & m) == t2) & ((w.z & m) == t2) & ((w.w & m) == t2);
}

template <typename U, int IPT>
struct CoopSmem {
    static constexpr int TILE = COOP_THREADS * IPT;
    static constexpr size_t al(size_t x) { return (x + 127) / 128 * 128; }
    static constexpr size_t kb_off = 0;                                          // [TILE] U
    static constexpr size_t sk_off = al(kb_off + (size_t)TILE * sizeof(U));      // [TILE] U staged
    static constexpr size_t cnt_off = al(sk_off + (size_t)TILE * sizeof(U));     // [16][256] u32
    static constexpr size_t bins_off = cnt_off + (size_t)COOP_WARPS * 256 * 4;   // [4][256] u32
    static constexpr size_t gbase_off = bins_off + 4 * 256 * 4;                  // [256] i32
    static constexpr size_t misc_off = gbase_off + 256 * 4;                      // [64] i32
    static constexpr size_t bytes = misc_off + 64 * 4;
};

__device__ __forceinline__ void fence_acq_rel_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

// Bounded grid barrier (all CTAs resident: a cooperative launch). `epoch`
// counts this CTA's barriers so far (warp 0 keeps it). Arrival: a release
// fence and one add to this CTA's counter; warp 0 then polls every counter
// (lane k reads counter k) until each holds epoch x its CTAs, and fences
// (acquire) before the CTA goes on. Returns false once any wait has run out.
__device__ __forceinline__ bool coop_barrier(CoopState* st, unsigned int& epoch, uint32_t limit, uint32_t* error,
                                             int* flag_s, bool arrive = true) {
    __syncthreads();
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        ++epoch;
        bool ok = __shfl_sync(0xffffffffu, (int)(ld_volatile_u32(&st->abort) == 0), 0) != 0;
        if (ok && lane == 0 && arrive) {
            fence_acq_rel_gpu();  // this CTA's writes before its arrival
            atomicAdd(&st->arrive[(blockIdx.x % COOP_CTRS) * COOP_CTR_STRIDE], 1u);
        }
        __syncwarp();
        const unsigned int mapped = lane < COOP_CTRS ? (gridDim.x + COOP_CTRS - 1 - lane) / COOP_CTRS : 0u;
        const unsigned int want = epoch * mapped;
        uint32_t spins = 0;
        while (ok) {
            const bool mine = lane >= COOP_CTRS || ld_volatile_u32(&st->arrive[lane * COOP_CTR_STRIDE]) >= want;
            if (__all_sync(0xffffffffu, mine)) break;
            if (__any_sync(0xffffffffu, lane == 0 && ld_volatile_u32(&st->abort) != 0)) {
                ok = false;
                break;
            }
            if (++spins > limit) {
                if (lane == 0) {
                    atomicOr(error, ERR_TIMEOUT);
                    atomicExch(&st->abort, 1u);
                }
                ok = false;
                break;
            }
        }
        fence_acq_rel_gpu();  // the others' writes before this CTA's reads
        if (lane == 0) *flag_s = ok ? 1 : 0;
    }
    __syncthreads();
    return *flag_s != 0;
}

// Exclusive prefix of v over the CTA's threads (COOP_THREADS); *total gets
// the sum. tmp: COOP_WARPS words of shared memory.
__device__ __forceinline__ uint32_t coop_exclusive_scan(uint32_t v, uint32_t* tmp, uint32_t* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) tmp[warp] = x;
    __syncthreads();
    uint32_t before = 0, all = 0;
#pragma unroll
    for (int w = 0; w < COOP_WARPS; ++w) {
        const uint32_t s = tmp[w];
        before += w < warp ? s : 0u;
        all += s;
    }
    __syncthreads();
    *total = all;
    return before + x - v;
}

// The keys [g, g + n) into shared memory, past L1 (other CTAs wrote them);
// from a 16-byte aligned source by 16-byte loads, all issued before the
// first store.
template <typename U, int TILE>
__device__ __forceinline__ void coop_load(U* kb, const U* g, int n, int tid) {
    constexpr int VN = 16 / (int)sizeof(U);
    constexpr int PER = (TILE / VN + COOP_THREADS - 1) / COOP_THREADS;
    int head = 0;
    if (((uintptr_t)g & 15) == 0) {
        const int nv = n / VN;
        const uint4* g4 = reinterpret_cast<const uint4*>(g);
        uint4* s4 = reinterpret_cast<uint4*>(kb);
        uint4 r[PER];
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            const int v = tid + k * COOP_THREADS;
            if (v < nv) r[k] = __ldcg(g4 + v);
        }
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            const int v = tid + k * COOP_THREADS;
            if (v < nv) s4[v] = r[k];
        }
        head = nv * VN;
    }
    for (int i = head + tid; i < n; i += COOP_THREADS) kb[i] = __ldcg(g + i);
}

// The keys of shared memory to [g, g + n), by 16-byte stores where g allows.
template <typename U>
__device__ __forceinline__ void coop_store(U* g, const U* kb, int n, int tid) {
    constexpr int VN = 16 / (int)sizeof(U);
    int head = 0;
    if (((uintptr_t)g & 15) == 0) {
        const int nv = n / VN;
        for (int v = tid; v < nv; v += COOP_THREADS)
            reinterpret_cast<uint4*>(g)[v] = reinterpret_cast<const uint4*>(kb)[v];
        head = nv * VN;
    }
    for (int i = head + tid; i < n; i += COOP_THREADS) g[i] = kb[i];
}

template <typename U, int XF, int IPT>
__global__ void __launch_bounds__(COOP_THREADS, 2) k_lsd_coop(CoopArgs<U> a) {
    static_assert(sizeof(U) == 2 || sizeof(U) == 4, "2- and 4-byte keys");
    using L = CoopSmem<U, IPT>;
    constexpr int TILE = L::TILE;
    static_assert(TILE <= (int)COOP_COUNT_MASK && (int)sizeof(U) < 8, "a tile's counts and pass tags fit 16 bits");
    constexpr int RADIX = 256;
    constexpr int ND = (int)sizeof(U);
    extern __shared__ __align__(128) unsigned char smem[];
    U* kb = reinterpret_cast<U*>(smem + L::kb_off);
    U* sk = reinterpret_cast<U*>(smem + L::sk_off);
    uint32_t* cnt = reinterpret_cast<uint32_t*>(smem + L::cnt_off);
    uint32_t* bins = reinterpret_cast<uint32_t*>(smem + L::bins_off);
    int* gbase = reinterpret_cast<int*>(smem + L::gbase_off);
    int* misc = reinterpret_cast<int*>(smem + L::misc_off);  // [0] barrier flag, [1] live count, [2..] digits
    uint32_t* tmp = reinterpret_cast<uint32_t*>(misc + 32);  // [16] scan scratch
    __shared__ unsigned long long red_diff[COOP_WARPS];
    __shared__ unsigned int red_flags[COOP_WARPS];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int t = blockIdx.x, T = gridDim.x;
    const size_t n = a.n;
    const size_t base = (size_t)t * TILE;
    const int tile_n = (int)min((size_t)TILE, n - base);
    const uint32_t lt = lanemask_lt();
    PeerMasks<8> pm;
    pm.init(lane);
    unsigned int epoch = 0;

    // ---- 0. the tile, what varies, sortedness, every digit's counts
    const U first = to_key<U, XF>(a.data[0]);
    zero_counters<COOP_WARPS * RADIX, COOP_THREADS>(cnt, tid);
    __syncthreads();
    unsigned long long diff = 0;
    unsigned int flags = 0;
    coop_load<U, TILE>(kb, a.data + base, tile_n, tid);
    __syncthreads();
    for (int i = tid; i < tile_n; i += COOP_THREADS) {
        const U k = to_key<U, XF>(kb[i]);
        kb[i] = k;
        diff |= (unsigned long long)(U)(k ^ first);
#pragma unroll
        for (int d = 0; d < ND; ++d) atomicAdd(&cnt[d * RADIX + ((k >> (8 * d)) & 255u)], 1u);
    }
    __syncthreads();
    for (int i = tid; i < tile_n; i += COOP_THREADS) {
        if (base + i == 0) continue;
        const U p = i > 0 ? kb[i - 1] : to_key<U, XF>(a.data[base - 1]);
        const U k = kb[i];
        flags |= p > k ? SCAN_NOT_ASC : 0u;
        flags |= p < k ? SCAN_NOT_DESC : 0u;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        diff |= __shfl_xor_sync(0xffffffffu, diff, o);
        flags |= __shfl_xor_sync(0xffffffffu, flags, o);
    }
    if (lane == 0) {
        red_diff[warp] = diff;
        red_flags[warp] = flags;
    }
    for (int i = tid; i < ND * RADIX; i += COOP_THREADS)
        if (cnt[i]) atomicAdd(&a.hist[i], cnt[i]);
    __syncthreads();
    if (tid == 0) {
        for (int w = 1; w < COOP_WARPS; ++w) {
            diff |= red_diff[w];
            flags |= red_flags[w];
        }
        if (diff) atomicOr(&a.st->diff, diff);
        if (flags) atomicOr(&a.st->flags, flags);
    }
    if (!coop_barrier(a.st, epoch, a.spin_limit, a.error, misc, !(a.withhold_cta0 && t == 0))) return;

    // the plan, the same in every CTA
    if (tid == 0) {
        const unsigned long long gd = ld_volatile_u64(&a.st->diff);
        const unsigned int gf = ld_volatile_u32(&a.st->flags);
        int mode = MODE_SORT;
        if (!(gf & SCAN_NOT_ASC)) mode = MODE_SORTED;
        else if (!(gf & SCAN_NOT_DESC)) mode = MODE_REVERSE;
        int m = 0;
        if (mode == MODE_SORT)
            for (int d = 0; d < ND; ++d)
                if (((gd >> (8 * d)) & 255ull) && ld_volatile_u32(&a.hist[d * RADIX + ((first >> (8 * d)) & 255u)]) < n)
                    misc[2 + m++] = d;
        misc[1] = mode == MODE_SORT ? m : -mode;
        if (t == 0) {
            a.plan->mode = mode;
            a.plan->n_live = m;
            for (int j = 0; j < m; ++j) a.plan->pass[j] = misc[2 + j];
            a.plan->divert_shift = 0;
        }
    }
    __syncthreads();
    if (t == 0) {  // each live digit's largest bucket, as the multi-launch plan reports it
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            uint32_t mx = tid < RADIX ? ld_volatile_u32(&a.hist[d * RADIX + tid]) : 0u;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
            if (lane == 0) tmp[warp] = mx;
            __syncthreads();
            if (tid == 0) {
                uint32_t all = 0;
                for (int w = 0; w < COOP_WARPS; ++w) all = max(all, tmp[w]);
                const unsigned long long gd = ld_volatile_u64(&a.st->diff);
                const bool live = ((gd >> (8 * d)) & 255ull) &&
                                  ld_volatile_u32(&a.hist[d * RADIX + ((first >> (8 * d)) & 255u)]) < n;
                a.maxb[d] = live ? all : 0ull;
            }
            __syncthreads();
        }
    }
    const int m = misc[1];
    if (m == -MODE_REVERSE) {  // descending input: reversed in place (pairs never span two CTAs' ranges)
        for (size_t i = base + tid; i < base + tile_n && i < n / 2; i += COOP_THREADS) {
            const U x = a.data[i];
            a.data[i] = a.data[n - 1 - i];
            a.data[n - 1 - i] = x;
        }
        return;
    }
    if (m <= 0) return;  // already sorted, or nothing varies

    // every digit's start in its histogram (the same in every CTA and pass)
    {
        uint32_t hv[ND];
#pragma unroll
        for (int d = 0; d < ND; ++d) hv[d] = tid < RADIX ? ld_volatile_u32(&a.hist[d * RADIX + tid]) : 0u;
        uint32_t total;
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            const uint32_t e = coop_exclusive_scan(hv[d], tmp, &total);
            if (tid < RADIX) bins[d * RADIX + tid] = e;
        }
    }

    const int wbase = warp * 32 * IPT + lane;
    for (int j = 0; j < m; ++j) {
        const int shift = 8 * misc[2 + j];
        const bool last = j == m - 1;
        U* dst = (j & 1) ? a.data : a.alt;
        auto dig = [&](U k) -> uint32_t { return __byte_perm((uint32_t)k, 0u, 0x4440u | (uint32_t)(shift >> 3)); };

        // ---- 1. the previous pass's output (written by other CTAs: past L1)
        if (j > 0) {
            if (!coop_barrier(a.st, epoch, a.spin_limit, a.error, misc)) return;
            const U* src = (j & 1) ? a.alt : a.data;
            coop_load<U, TILE>(kb, src + base, tile_n, tid);
            zero_counters<COOP_WARPS * RADIX, COOP_THREADS>(cnt, tid);
        } else {
            zero_counters<COOP_WARPS * RADIX, COOP_THREADS>(cnt, tid);
        }
        __syncthreads();

        // ---- 2. per-warp counts, the tile's counts, tile-local starts, ranks
#pragma unroll
        for (int i = 0; i < IPT; ++i) {
            const int idx = wbase + i * 32;
            if (idx < tile_n) atomicAdd(&cnt[warp * RADIX + dig(kb[idx])], 1u);
        }
        __syncthreads();
        uint32_t tc = 0;
        if (tid < RADIX) {
#pragma unroll
            for (int w = 0; w < COOP_WARPS; ++w) {
                const uint32_t c = cnt[w * RADIX + tid];
                cnt[w * RADIX + tid] = tc;
                tc += c;
            }
            a.tcnt[(size_t)t * RADIX + tid] = (unsigned short)((unsigned)(j + 1) << COOP_COUNT_BITS | tc);
        }
        uint32_t total;
        const uint32_t lstart = coop_exclusive_scan(tc, tmp, &total);
        if (tid < RADIX) {
#pragma unroll
            for (int w = 0; w < COOP_WARPS; ++w) cnt[w * RADIX + tid] += lstart;
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < IPT; ++i) {
            const int idx = wbase + i * 32;
            const bool valid = idx < tile_n;
            const U k = kb[valid ? idx : 0];
            const uint32_t d = dig(k);
            uint32_t peers = (i % 3 == 0) ? __match_any_sync(0xffffffffu, d) : pm.peers(d);
            peers &= __ballot_sync(0xffffffffu, valid);
            if (valid) {
                const uint32_t c = cnt[warp * RADIX + d];
                cnt[warp * RADIX + d] = c + __popc(peers);
                sk[c + __popc(peers & lt)] = k;
            }
            __syncwarp();
        }

        // ---- 3. each digit's keys in earlier tiles: the sum of their
        // published counts. Thread (g, q) reads uint4 column q (digits 8q ..
        // 8q + 7) of rows g, g + 16, ..., re-reading a word until all of its
        // fields carry this pass's tag; the 16 row groups meet in the counters.
        {
            const int q = tid & 31, g = tid >> 5;
            const uint4* rows = reinterpret_cast<const uint4*>(a.tcnt);
            const unsigned int tag = (unsigned int)(j + 1);
            uint32_t part[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            bool ok = true;
            uint32_t spins = 0;
            constexpr int INFLIGHT = 6;
            for (int r0 = g; r0 < t && ok; r0 += 16 * INFLIGHT) {
                uint4 v[INFLIGHT];
#pragma unroll
                for (int u = 0; u < INFLIGHT; ++u) {
                    const int r = r0 + 16 * u;
                    if (r < t) v[u] = __ldcv(rows + (size_t)r * 32 + q);
                }
#pragma unroll
                for (int u = 0; u < INFLIGHT; ++u) {
                    const int r = r0 + 16 * u;
                    if (r >= t || !ok) continue;
                    while (!coop_tagged(v[u], tag)) {
                        if (++spins > a.spin_limit) {
                            ok = false;
                            break;
                        }
                        v[u] = __ldcv(rows + (size_t)r * 32 + q);
                    }
                    const uint32_t w[4] = {v[u].x, v[u].y, v[u].z, v[u].w};
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        part[2 * e] += w[e] & COOP_COUNT_MASK;
                        part[2 * e + 1] += (w[e] >> 16) & COOP_COUNT_MASK;
                    }
                }
            }
            if (!ok) {
                atomicOr(a.error, ERR_TIMEOUT);
                atomicExch(&a.st->abort, 1u);
            }
            if (__syncthreads_or(!ok)) return;
#pragma unroll
            for (int e = 0; e < 8; ++e) cnt[g * RADIX + 8 * q + e] = part[e];
            __syncthreads();
        }

        // ---- 4. global starts, then runs per digit
        if (tid < RADIX) {
            uint32_t before = 0;
#pragma unroll
            for (int g = 0; g < COOP_WARPS; ++g) before += cnt[g * RADIX + tid];
            gbase[tid] = (int)(bins[misc[2 + j] * RADIX + tid] + before) - (int)lstart;
        }
        __syncthreads();
        for (int s = tid; s < tile_n; s += COOP_THREADS) {
            const U k = sk[s];
            const int p = gbase[dig(k)] + s;
            if ((size_t)(unsigned)p < n) dst[p] = last ? from_key<U, XF>(k) : k;
            else atomicOr(a.error, ERR_BOUNDS);
        }
    }
    if (m & 1) {  // the last pass wrote the scratch: copy back
        if (!coop_barrier(a.st, epoch, a.spin_limit, a.error, misc)) return;
        coop_load<U, TILE>(kb, a.alt + base, tile_n, tid);
        __syncthreads();
        coop_store<U>(a.data + base, kb, tile_n, tid);
    }
}

}  // namespace ts
