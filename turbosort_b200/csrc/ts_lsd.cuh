// ts_lsd.cuh — the LSD radix sort kernels.
//
//   k_scan      one read (early exit): bits that vary (src/radix/histogram.rs:55-68)
//               and whether the input is already sorted either way
//               (src/presorted.rs:15-65)
//   k_hist      one read: histograms of every varying digit
//               (src/radix/histogram.rs:15-110)
//               and, in its last CTA to finish, the plan: live passes
//               (src/radix/mod.rs:229-239), diverting, and the exclusive scans
//               (src/radix/prefix_sum.rs:17-24), decided on the device
//   k_onesweep  one stable scatter pass per live digit
//               (src/radix/scatter.rs:26-247): warp ranking with match.any,
//               decoupled look-back across tiles, the tile reordered in shared
//               memory so that global writes are runs per digit. The key
//               transform (src/key.rs:135-197) is fused into the first load
//               and the last store. Optionally carries a u32 position (the
//               stable order() of src/by_key.rs:254-310).
//   k_finish_keys  copy-back for an odd pass count (src/radix/mod.rs:265-267)
//               or the reversal of descending input; k_iota_if_unsorted, the
//               order of an input that needed no pass
#pragma once

#include <type_traits>

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
// k_scan: OR of (key ^ first key) and the two sortedness flags. CTAs leave
// as soon as every digit has varied and both directions are disproved,
// which random input does in its first chunk.
// ---------------------------------------------------------------------------
template <typename U, int XF, int THREADS>
__global__ void __launch_bounds__(THREADS) k_scan(const U* __restrict__ src, size_t n, int bits, int nd,
                                                  ScanState* __restrict__ st, int vec_ok, uint4* __restrict__ lb,
                                                  size_t lb_vecs) {
    dep_release();  // the histogram kernel may launch early (it waits for this one)
    // the first onesweep launch's look-back region starts at zero (each
    // launch clears the next one's); done before any warp can leave
    for (size_t i = (size_t)blockIdx.x * THREADS + threadIdx.x; i < lb_vecs; i += (size_t)gridDim.x * THREADS)
        lb[i] = make_uint4(0u, 0u, 0u, 0u);
    using V = Vec16<U>;
    constexpr int VN = V::N;
    constexpr int UNROLL = 4;
    __shared__ unsigned long long s_diff[THREADS / 32];
    __shared__ unsigned s_flags[THREADS / 32];
    __shared__ int s_stop;
    const U first = to_key<U, XF>(src[0]);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
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
        // merge over the CTA (every warp runs the same iterations), then one
        // thread reads the global state and publishes only what it lacks: once
        // the input is known to be unsorted with every digit varying, CTAs
        // leave without touching the two shared words (thousands of atomics
        // on one address would serialise)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            diff |= __shfl_xor_sync(0xffffffffu, diff, o);
            flags |= __shfl_xor_sync(0xffffffffu, flags, o);
        }
        if (lane == 0) {
            s_diff[warp] = diff;
            s_flags[warp] = flags;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int w = 0; w < THREADS / 32; ++w) {
                diff |= s_diff[w];
                flags |= s_flags[w];
            }
            unsigned long long g = ld_volatile_u64(&st->diff);
            unsigned gf = ld_volatile_u32(&st->flags);
            if (diff & ~(published | g)) {
                atomicOr(&st->diff, diff);
                g |= diff;
            }
            if (flags & ~(pub_flags | gf)) {
                atomicOr(&st->flags, flags);
                gf |= flags;
            }
            published |= diff;
            pub_flags |= flags;
            s_stop = (gf == (SCAN_NOT_ASC | SCAN_NOT_DESC)) && all_digits_vary(g, bits, nd);
        }
        __syncthreads();
        if (s_stop) return;
    }
}

// ---------------------------------------------------------------------------
// k_hist: histograms of the varying digits in one read. Each lane counts
// into its own copy, and the copy index is the fastest-moving, so the 32
// lanes of a warp always hit 32 different banks (no conflicts, no shared
// addresses) whatever the digits are.
// ---------------------------------------------------------------------------
template <int RADIX, int ND>
__host__ __device__ constexpr int hist_copies() {
    return RADIX <= 256 ? (ND <= 4 ? 32 : 16) : 1;
}

template <typename U, int XF, int BITS, bool DIVERT>
__device__ void plan_body(const U* __restrict__ src, size_t n, const ScanState* __restrict__ st,
                          const unsigned long long* ghist, unsigned long long* __restrict__ bins,
                          Plan* __restrict__ plan, int stable, unsigned long long* __restrict__ maxb_out,
                          int divert);

template <typename U, int XF, int BITS, int THREADS, bool DIVERT>
__global__ void __launch_bounds__(THREADS) k_hist(const U* __restrict__ src, size_t n, ScanState* __restrict__ st,
                                                  unsigned long long* __restrict__ ghist, int vec_ok,
                                                  unsigned long long* __restrict__ bins, Plan* __restrict__ plan,
                                                  int stable, unsigned long long* __restrict__ maxb_out,
                                                  int divert) {
    dep_wait();
    dep_release();
    static_assert(THREADS >= 32 * ((Bits<U>::W + BITS - 1) / BITS), "the plan scans a digit a warp");
    constexpr int RADIX = 1 << BITS;
    constexpr int ND = (Bits<U>::W + BITS - 1) / BITS;
    constexpr int COPIES = hist_copies<RADIX, ND>();
    using V = Vec16<U>;
    constexpr int VN = V::N;
    constexpr int UNROLL = 4;
    extern __shared__ __align__(16) uint32_t h_s[];  // [ND][RADIX][COPIES]
    const unsigned long long diff = st->diff;
    uint32_t counted = 0;
#pragma unroll
    for (int d = 0; d < ND; ++d)
        if ((diff >> (d * BITS)) & (unsigned long long)(RADIX - 1)) counted |= 1u << d;
    for (int i = threadIdx.x; i < ND * RADIX * COPIES; i += THREADS) h_s[i] = 0;
    __syncthreads();
    uint32_t* my_h = h_s + threadIdx.x % COPIES;
    // one key into every counted digit's histogram; ALL: no digit is skipped
    auto count = [&](U raw, auto all_tag) {
        constexpr bool ALL = decltype(all_tag)::value;
        const U key = to_key<U, XF>(raw);
#pragma unroll
        for (int d = 0; d < ND; ++d)
            if (ALL || (counted & (1u << d)))
                atomicAdd(&my_h[(d * RADIX + digit_of(key, d * BITS, RADIX - 1)) * COPIES], 1u);
    };
    auto sweep = [&](auto all_tag) {
        const size_t nvec = vec_ok ? n / VN : 0;
        const size_t stride = (size_t)gridDim.x * THREADS;
        const uint4* v4 = reinterpret_cast<const uint4*>(src);
        for (size_t v0 = (size_t)blockIdx.x * THREADS + threadIdx.x; v0 < nvec; v0 += stride * UNROLL) {
            V x[UNROLL];
#pragma unroll
            for (int u = 0; u < UNROLL; ++u)
                if (v0 + u * stride < nvec) x[u].v = __ldcs(v4 + v0 + u * stride);
#pragma unroll
            for (int u = 0; u < UNROLL; ++u)
                if (v0 + u * stride < nvec) {
#pragma unroll
                    for (int e = 0; e < VN; ++e) count(x[u].e[e], all_tag);
                }
        }
        for (size_t i = nvec * VN + (size_t)blockIdx.x * THREADS + threadIdx.x; i < n; i += stride)
            count(src[i], all_tag);
    };
    if (counted == (1u << ND) - 1) sweep(std::true_type{});
    else sweep(std::false_type{});
    __syncthreads();
    for (int i = threadIdx.x; i < ND * RADIX; i += THREADS) {
        uint32_t s = 0;
#pragma unroll
        for (int c = 0; c < COPIES; ++c) s += h_s[i * COPIES + ((c + i) & (COPIES - 1))];
        if (s) atomicAdd(&ghist[i], (unsigned long long)s);
    }
    // the last CTA to finish makes the plan (one launch fewer than a
    // separate plan kernel): its ticket comes after every other CTA's counts
    __shared__ int last_s;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last_s = atomicAdd(&st->hist_done, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last_s) return;
    __threadfence();
    plan_body<U, XF, BITS, DIVERT>(src, n, st, ghist, bins, plan, stable, maxb_out, divert);
}

// ---------------------------------------------------------------------------
// Diverting (src/radix/divert.rs:38-54, :95-104): how many of the lowest
// live digits need no pass, because the digits above them already split the
// keys into runs short enough to finish by a direct sort of each run.
// ---------------------------------------------------------------------------
constexpr int DIVERT_SLACK_BITS = 2;  // divert.rs:19
constexpr int DIVERT_MIN_SKIP = 3;    // divert.rs:28

// log2(x) in eighths of a bit, never above the true value (divert.rs:95-104)
__host__ __device__ inline unsigned log2_eighths(unsigned long long x) {
    int ip = 63;
    while (ip > 0 && !((x >> ip) & 1ull)) --ip;
    const unsigned long long frac = ip >= 3 ? (x >> (ip - 3)) & 7ull : (x << (3 - ip)) & 7ull;
    return 8u * (unsigned)ip + (unsigned)frac;
}

// max_bucket[i]: the largest bucket of the i-th live digit, least significant first
__host__ __device__ inline int skippable_digits(int n_live, unsigned long long len,
                                                const unsigned long long* max_bucket) {
    const unsigned log_len = log2_eighths(len);
    const unsigned need = log_len + 8u * DIVERT_SLACK_BITS;
    unsigned have = 0;
    for (int i = n_live - 1; i >= DIVERT_MIN_SKIP; --i) {
        have += log_len - log2_eighths(max_bucket[i]);
        if (have >= need) return i;
    }
    return 0;
}

// ---------------------------------------------------------------------------
// The plan, by one CTA of at least 32 * ND threads (k_hist's last). Live
// passes are the counted digits whose histogram does
// not hold every key in the first key's bucket; each gets its exclusive scan.
// `stable` (sort_by_key) leaves descending input to the passes, since a
// plain reversal would reverse equal keys. With DIVERT (keys only) the
// lowest live digits are left out when diverting.rs's rule allows it
// (src/radix/mod.rs:240-242), and divert_shift tells the finishing kernels
// which runs remain.
// ---------------------------------------------------------------------------
template <typename U, int XF, int BITS, bool DIVERT>
__device__ void plan_body(const U* __restrict__ src, size_t n, const ScanState* __restrict__ st,
                          const unsigned long long* ghist, unsigned long long* __restrict__ bins,
                          Plan* __restrict__ plan, int stable, unsigned long long* __restrict__ maxb_out,
                          int divert) {
    constexpr int RADIX = 1 << BITS;
    constexpr int ND = (Bits<U>::W + BITS - 1) / BITS;
    __shared__ int live_s[ND];
    __shared__ unsigned long long max_s[ND];
    const U first = to_key<U, XF>(src[0]);
    const unsigned long long diff = st->diff;
    if (threadIdx.x < ND) {
        const int d = threadIdx.x;
        const bool counted = ((diff >> (d * BITS)) & (unsigned long long)(RADIX - 1)) != 0;
        live_s[d] = counted && __ldcg(&ghist[(size_t)d * RADIX + digit_of(first, d * BITS, RADIX - 1)]) < n;
    }
    __syncthreads();
    // warp w scans digit w's histogram
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp < ND && live_s[warp]) {
        unsigned long long carry = 0, mx = 0;
        for (int r0 = 0; r0 < RADIX; r0 += 32) {
            const int r = r0 + lane;
            unsigned long long v = r < RADIX ? __ldcg(&ghist[(size_t)warp * RADIX + r]) : 0ull;
            mx = v > mx ? v : mx;
            unsigned long long x = v;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            if (r < RADIX) bins[(size_t)warp * RADIX + r] = carry + x - v;
            carry += __shfl_sync(0xffffffffu, x, 31);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long y = __shfl_xor_sync(0xffffffffu, mx, o);
            mx = y > mx ? y : mx;
        }
        if (lane == 0) max_s[warp] = mx;
    }
    __syncthreads();
    // each digit's largest bucket (0: not live), for callers that estimate
    // what a sort of more keys from the same distribution would do
    if (threadIdx.x < ND) maxb_out[threadIdx.x] = live_s[threadIdx.x] ? max_s[threadIdx.x] : 0ull;
    if (threadIdx.x == 0) {
        const unsigned f = st->flags;
        int mode = MODE_SORT;
        if (!(f & SCAN_NOT_ASC)) mode = MODE_SORTED;
        else if (!stable && !(f & SCAN_NOT_DESC)) mode = MODE_REVERSE;
        int live[ND];
        unsigned long long maxb[ND];
        int m = 0;
        if (mode == MODE_SORT)
            for (int d = 0; d < ND; ++d)
                if (live_s[d]) {
                    maxb[m] = max_s[d];
                    live[m++] = d;
                }
        int skip = 0;
        if constexpr (DIVERT) {
            if (divert && !stable && mode == MODE_SORT) skip = skippable_digits(m, n, maxb);
        }
        for (int i = skip; i < m; ++i) plan->pass[i - skip] = live[i];
        plan->n_live = m - skip;
        plan->divert_shift = skip > 0 ? live[skip] * BITS : 0;
        plan->mode = mode;
    }
}


// ---------------------------------------------------------------------------
// Finishing kernels, each a no-op unless the plan calls for it.
// ---------------------------------------------------------------------------
// The end of a key sort, in one launch: the copy back for an odd count of
// live passes (src/radix/mod.rs:265-267), or the reversal of descending
// input (src/presorted.rs:15-65), as the plan says; nothing otherwise.
template <typename U>
__global__ void k_finish_keys(const Plan* __restrict__ plan, const U* from, U* to, size_t n, int vec_ok) {
    dep_wait();
    dep_release();
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    if (plan->mode == MODE_REVERSE) {
        for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n / 2; i += stride) {
            const U x = to[i];
            to[i] = to[n - 1 - i];
            to[n - 1 - i] = x;
        }
        return;
    }
    if (plan->mode != MODE_SORT || (plan->n_live & 1) == 0) return;
    using V = Vec16<U>;
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

static __global__ void k_iota_if_unsorted(const Plan* __restrict__ plan, uint32_t* __restrict__ order, size_t n) {
    dep_wait();
    dep_release();
    if (plan->mode == MODE_SORT && plan->n_live > 0) return;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) order[i] = (uint32_t)i;
}

}  // namespace ts
