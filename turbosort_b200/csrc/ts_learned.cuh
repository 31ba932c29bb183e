// ts_learned.cuh — the learned MSD partition: a two-level piecewise-linear
// CDF model of the keys, fitted on the GPU to a sample whose exact ranks come
// from the plain radix sort, maps each key to one of B buckets in one
// partition pass; the segmented sort then sorts every bucket.
//
// The model only chooses positions. The bucket map is non-decreasing in the
// key by construction (every stage is monotone and clamped, whatever the
// parameters hold), so equal keys share a bucket and every key of bucket b
// precedes every key of bucket b + 1: sorting the buckets gives exactly the
// plain sort's output.
//
// All arithmetic is on radix keys (the order-preserving unsigned images).
//   root    L + 1 knots at the sample's quantiles r/L, compared on a 32-bit
//           prefix of (key - kmin) (a monotone image): the knot segment a key
//           falls in is its leaf j, and the root's CDF there is r/L.
//   leaf j  t = (key - klo_j) / (khi_j - klo_j) in [0, 1] in the leaf's own
//           range (full key precision: one leaf spans a narrow key range);
//           a P-piece linear CDF through breakpoints bp_0 = 0 <= ... <= bp_P = 1
//           placed at the leaf's sample quantiles, with heights v_0..v_P that
//           gradient descent fits (Adam on the mean squared rank error);
//           y = y0_j + h_j * PL_j(t), bucket = floor(y * B) clamped into the
//           piece's and then the leaf's bucket range [lo_j, hi_j].
#pragma once

#include "ts_common.cuh"
#include "ts_segmented.cuh"

namespace ts {

constexpr int LM_P = 8;                // pieces per leaf
constexpr int LM_MAX_LEAVES = 2048;
constexpr int LM_TRAIN_THREADS = 256;

struct LmHead {
    unsigned long long kmin, kmax;  // radix keys of the sample's extremes
    float inv_range;                // 1 / (kmax - kmin), for the no-model ablation
    int shift;                      // prefix = (key - kmin) >> shift fits 32 bits
    int leaves;
    int buckets;
    int use_model;                  // 0: equal-width buckets over [kmin, kmax] (no model)
    int pad;
};

// per-leaf packed record for the partition kernels (one 16-byte load)
struct __align__(16) LmLeaf {
    unsigned long long klo;  // radix key of the leaf's first sample
    float winv;              // 1 / (khi - klo), 0 when the leaf's samples are all equal
    short lo, hi;            // the leaf's bucket range
};

// device tables of a fitted model
struct LmTables {
    uint32_t* rootk;  // [2^depth] root knots (prefixes), Eytzinger order
    LmLeaf* leaf;     // [L]
    float* bp;        // [L * (P - 1)] interior breakpoints of each leaf
    float* c;         // [L * (P + 1)] bucket-space heights, non-decreasing per leaf
    float* v;         // [L * (P + 1)] trained heights, leaf units
    float* y0;        // [L] leaf's first rank / m
    float* h;         // [L] leaf's share of the ranks
    int* first;       // [L] the leaf's samples: [first, last], -1 when empty
    int* last;
};

__host__ __device__ inline LmHead lm_make_head(unsigned long long kmin, unsigned long long kmax, int leaves,
                                               int buckets, int use_model) {
    LmHead h{};
    h.kmin = kmin;
    h.kmax = kmax;
    const unsigned long long r = kmax > kmin ? kmax - kmin : 0ull;
    int bits = 0;
    while (bits < 64 && (r >> bits) != 0ull) ++bits;
    h.shift = bits > 32 ? bits - 32 : 0;
    h.inv_range = r ? 1.f / (float)r : 0.f;
    h.leaves = leaves;
    h.buckets = buckets;
    h.use_model = use_model;
    return h;
}

template <typename U>
__device__ __forceinline__ uint32_t lm_prefix(const LmHead& m, U key) {
    unsigned long long k = (unsigned long long)key;
    if (k <= m.kmin) return 0u;
    if (k > m.kmax) k = m.kmax;
    return (uint32_t)((k - m.kmin) >> m.shift);
}

// Depth of the root's search tree: 2^depth - 1 >= leaves - 1 interior knots.
__host__ __device__ inline int lm_depth(int leaves) {
    int d = 0;
    while ((1 << d) < leaves) ++d;
    return d;
}

// The leaf of prefix p: the number of interior knots <= p, found in the
// knots' Eytzinger (breadth-first) layout E[1 .. 2^depth - 1] (padding
// UINT32_MAX), so the first five levels of every search read five distinct
// 32-word-aligned rows and the lanes of a warp do not collide on banks.
__device__ __forceinline__ int lm_root(const uint32_t* E, int leaves, int depth, uint32_t p) {
    int i = 1;
    for (int s = 0; s < depth; ++s) i = 2 * i + (E[i] <= p ? 1 : 0);
    return min(i - (1 << depth), leaves - 1);
}

// t in [0, 1]: the key's place in the leaf's sample range.
template <typename U>
__device__ __forceinline__ float lm_t(U key, unsigned long long klo, float winv) {
    const unsigned long long k = (unsigned long long)key;
    if (k <= klo) return 0.f;
    return fminf(1.f, __ull2float_rn(k - klo) * winv);
}

// Piece of t among non-decreasing interior breakpoints bp[0..P-2]: k = the
// number of them <= t, and t's fraction inside piece k.
__device__ __forceinline__ void lm_piece(const float* bp, float t, int& k, float& frac) {
    static_assert(LM_P == 8, "the search below covers 7 interior breakpoints");
    k = 0;
    if (bp[3] <= t) k = 4;
    if (bp[k + 1] <= t) k += 2;
    if (bp[k] <= t) k += 1;
    const float left = k == 0 ? 0.f : bp[k - 1];
    const float right = k == LM_P - 1 ? 1.f : bp[k];
    frac = right > left ? fminf(1.f, __fdividef(t - left, right - left)) : 0.f;
}

// ---- sample and fit -----------------------------------------------------------
template <typename U>
__global__ void k_lm_sample(const U* __restrict__ src, size_t n, size_t every, U* __restrict__ out, size_t m,
                            int xf_kind) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
        const U v = src[i * every + every / 2 < n ? i * every + every / 2 : n - 1];
        out[i] = xf_kind == 0 ? v : (xf_kind == 1 ? to_key<U, 1>(v) : to_key<U, 2>(v));
    }
}

// Root knots at the sorted sample's quantiles (kept non-decreasing whatever
// the sample holds), stored in Eytzinger order; the model header. One CTA of
// 1024 threads.
template <typename U>
__global__ void __launch_bounds__(1024) k_lm_root(const U* __restrict__ s, size_t m, int leaves, int buckets,
                                                  int use_model, LmHead* __restrict__ head, uint32_t* __restrict__ E) {
    __shared__ uint32_t kn[LM_MAX_LEAVES + 1];
    const LmHead hd = lm_make_head((unsigned long long)s[0], (unsigned long long)s[m - 1], leaves, buckets, use_model);
    for (int r = threadIdx.x; r <= leaves; r += blockDim.x) {
        const size_t idx = r == leaves ? m - 1 : min(m - 1, (size_t)((double)r * (double)m / leaves));
        kn[r] = r == 0 ? 0u : lm_prefix(hd, s[idx]);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int r = 1; r <= leaves; ++r) kn[r] = max(kn[r], kn[r - 1]);
        *head = hd;
    }
    __syncthreads();
    // node i (level l = floor(log2 i), position q = i - 2^l) holds interior
    // knot number (2q + 1) 2^(depth-1-l) - 1 in sorted order, i.e. kn[that + 1]
    const int depth = lm_depth(leaves);
    for (int i = threadIdx.x; i < (1 << depth); i += blockDim.x) {
        if (i == 0) {
            E[0] = 0u;
            continue;
        }
        const int l = 31 - __clz(i);
        const int r = (2 * (i - (1 << l)) + 1) * (1 << (depth - 1 - l)) - 1;
        E[i] = r < leaves - 1 ? kn[r + 1] : 0xffffffffu;
    }
}

// The first and last sample of every leaf (each leaf's samples are contiguous:
// the sample is sorted and the root monotone). first / last start at -1.
template <typename U>
__global__ void k_lm_leaves(const U* __restrict__ s, size_t m, const LmHead* __restrict__ head,
                            const uint32_t* __restrict__ rootk, int* __restrict__ first, int* __restrict__ last) {
    const LmHead hd = *head;
    const int depth = lm_depth(hd.leaves);
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
        const int j = lm_root(rootk, hd.leaves, depth, lm_prefix(hd, s[i]));
        const int jp = i > 0 ? lm_root(rootk, hd.leaves, depth, lm_prefix(hd, s[i - 1])) : -1;
        const int jn = i + 1 < m ? lm_root(rootk, hd.leaves, depth, lm_prefix(hd, s[i + 1])) : -1;
        if (jp != j) first[j] = (int)i;
        if (jn != j) last[j] = (int)i;
    }
}

// Leaf ranges, breakpoints at the leaf's sample quantiles q/P, and the start
// of training: heights v_q = q/P, the sample's own CDF at the breakpoints
// (linear interpolation between them), which the fit then moves to the
// heights of least squared rank error over all the leaf's samples.
template <typename U>
__global__ void k_lm_init(const U* __restrict__ s, size_t m, int leaves, LmTables T) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < leaves; j += gridDim.x * blockDim.x) {
        const int f = T.first[j], l = T.last[j];
        LmLeaf lf{};
        float* bp = T.bp + (size_t)j * (LM_P - 1);
        float* v = T.v + (size_t)j * (LM_P + 1);
        if (f < 0) {
            lf.klo = 0;
            lf.winv = 0.f;
            for (int q = 0; q < LM_P - 1; ++q) bp[q] = 1.f;
            for (int q = 0; q <= LM_P; ++q) v[q] = 0.f;
            T.y0[j] = 0.f;
            T.h[j] = 0.f;
        } else {
            const unsigned long long klo = (unsigned long long)s[f], khi = (unsigned long long)s[l];
            lf.klo = klo;
            lf.winv = khi > klo ? 1.f / __ull2float_rn(khi - klo) : 0.f;
            const int cnt = l - f + 1;
            float prev = 0.f;
            for (int q = 1; q < LM_P; ++q) {
                const int idx = f + (int)(((long long)q * (cnt - 1) + LM_P / 2) / LM_P);
                const float t = fmaxf(prev, lm_t(s[idx], klo, lf.winv));
                bp[q - 1] = t;
                prev = t;
            }
            for (int q = 0; q <= LM_P; ++q) v[q] = (float)q / (float)LM_P;
            T.y0[j] = (float)((double)f / (double)m);
            T.h[j] = (float)((double)cnt / (double)m);
        }
        T.leaf[j] = lf;
    }
}

// One leaf's prediction (global CDF units) at leaf position t.
__device__ __forceinline__ float lm_predict(const float* bp, const float* pv, float y0, float h, float t, int& k,
                                            float& frac) {
    lm_piece(bp, t, k, frac);
    return fmaf(h, fmaf(pv[k + 1] - pv[k], frac, pv[k]), y0);
}

// dL/dv_q of L = (1/m) sum_i R_i^2, R_i = prediction_i - y_i, over one leaf's
// samples [f, l] (t_i and y_i from the callbacks), reduced over the block into
// g[0..P] of thread 0, with sum R^2 and max |R|.
template <typename TF, typename YF>
__device__ void lm_leaf_grads(int f, int l, const float* bp, const float* pv, float y0, float h, float inv_m,
                              TF t_of, YF y_of, float* g_red /* smem [warps][P+1] */, float* e_red /* [warps][2] */,
                              float (&g)[LM_P + 1], float& sse, float& emax) {
    float acc[LM_P + 1];
#pragma unroll
    for (int q = 0; q <= LM_P; ++q) acc[q] = 0.f;
    float s2 = 0.f, mx = 0.f;
    for (int i = f + (int)threadIdx.x; i <= l; i += blockDim.x) {
        int k;
        float frac;
        const float pred = lm_predict(bp, pv, y0, h, t_of(i), k, frac);
        const float r = pred - y_of(i);
        s2 = fmaf(r, r, s2);
        mx = fmaxf(mx, fabsf(r));
        const float gr = 2.f * inv_m * r * h;
#pragma unroll
        for (int q = 0; q < LM_P; ++q)
            if (q == k) {
                acc[q] = fmaf(gr, 1.f - frac, acc[q]);
                acc[q + 1] = fmaf(gr, frac, acc[q + 1]);
            }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
#pragma unroll
    for (int q = 0; q <= LM_P; ++q)
        for (int o = 16; o > 0; o >>= 1) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], o);
    for (int o = 16; o > 0; o >>= 1) {
        s2 += __shfl_xor_sync(0xffffffffu, s2, o);
        mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q <= LM_P; ++q) g_red[warp * (LM_P + 1) + q] = acc[q];
        e_red[warp * 2] = s2;
        e_red[warp * 2 + 1] = mx;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q <= LM_P; ++q) {
            float t = 0.f;
            for (int w = 0; w < warps; ++w) t += g_red[w * (LM_P + 1) + q];
            g[q] = t;
        }
        float ts = 0.f, tm = 0.f;
        for (int w = 0; w < warps; ++w) {
            ts += e_red[w * 2];
            tm = fmaxf(tm, e_red[w * 2 + 1]);
        }
        sse = ts;
        emax = tm;
    }
    __syncthreads();
}

// Training: one CTA per leaf (a leaf's heights only enter its own samples'
// terms of the loss, so leaves train independently), every Adam step on chip.
// Adam sees dL/dv scaled by m / (2 h^2), a per-leaf constant, which leaves its
// steps unchanged and keeps them clear of its epsilon. The step size is lr
// times the leaf's initial RMS rank error (in leaf units) and decays linearly
// to zero. Reports the loss before the first step and after the
// last, and the largest |rank error| after the last.
template <typename U>
__global__ void __launch_bounds__(LM_TRAIN_THREADS) k_lm_train(const U* __restrict__ s, size_t m, LmTables T,
                                                               int iters, float lr, double* __restrict__ loss_first,
                                                               double* __restrict__ loss_last,
                                                               float* __restrict__ max_err) {
    __shared__ float bp[LM_P - 1], pv[LM_P + 1];
    __shared__ float g_red[(LM_TRAIN_THREADS / 32) * (LM_P + 1)], e_red[(LM_TRAIN_THREADS / 32) * 2];
    const int j = blockIdx.x;
    const int f = T.first[j], l = T.last[j];
    if (f < 0 || l < f || (size_t)l >= m) return;  // empty leaf; uniform per CTA
    const LmLeaf lf = T.leaf[j];
    const float y0 = T.y0[j], h = T.h[j];
    const float inv_m = 1.f / (float)m;
    if (threadIdx.x < LM_P - 1) bp[threadIdx.x] = T.bp[(size_t)j * (LM_P - 1) + threadIdx.x];
    if (threadIdx.x <= LM_P) pv[threadIdx.x] = T.v[(size_t)j * (LM_P + 1) + threadIdx.x];
    __syncthreads();
    auto t_of = [&](int i) { return lm_t(s[i], lf.klo, lf.winv); };
    auto y_of = [&](int i) { return (float)(((double)i + 0.5) / (double)m); };
    const float scale = h > 0.f ? 0.5f * (float)m / (h * h) : 0.f;
    float m1 = 0.f, m2 = 0.f;  // Adam moments of height threadIdx.x (threads 0..P)
    float g[LM_P + 1];
    float sse = 0.f, emax = 0.f;
    const float b1 = 0.9f, b2 = 0.999f;
    __shared__ float rms0;  // the leaf's RMS rank error before training, in leaf units
    for (int it = 0; it < iters; ++it) {
        lm_leaf_grads(f, l, bp, pv, y0, h, inv_m, t_of, y_of, g_red, e_red, g, sse, emax);
        if (threadIdx.x == 0) {
            if (it == 0) {
                atomicAdd(loss_first, (double)sse / (double)m);
                rms0 = h > 0.f ? sqrtf(sse / (float)(l - f + 1)) / h : 0.f;
            }
#pragma unroll
            for (int q = 0; q <= LM_P; ++q) g_red[q] = g[q];  // hand the gradient to threads 0..P
        }
        __syncthreads();
        if (threadIdx.x <= LM_P) {
            const float gq = g_red[threadIdx.x] * scale;
            m1 = b1 * m1 + (1.f - b1) * gq;
            m2 = b2 * m2 + (1.f - b2) * gq * gq;
            const float c1 = 1.f - __powf(b1, (float)(it + 1)), c2 = 1.f - __powf(b2, (float)(it + 1));
            // steps start at lr x the leaf's RMS error (the scale of the corrections
            // it needs) and decay linearly to zero
            const float step = lr * rms0 * (1.f - (float)it / (float)iters);
            pv[threadIdx.x] -= step * (m1 / c1) / (sqrtf(m2 / c2) + 1e-8f);
        }
        __syncthreads();
    }
    lm_leaf_grads(f, l, bp, pv, y0, h, inv_m, t_of, y_of, g_red, e_red, g, sse, emax);
    if (threadIdx.x == 0) {
        if (iters == 0) atomicAdd(loss_first, (double)sse / (double)m);
        atomicAdd(loss_last, (double)sse / (double)m);
        atomicMax(reinterpret_cast<unsigned int*>(max_err), __float_as_uint(emax));
    }
    if (threadIdx.x <= LM_P) T.v[(size_t)j * (LM_P + 1) + threadIdx.x] = pv[threadIdx.x];
}

// The gradient alone, for checking the backward arithmetic against a float64
// oracle: leaf j's samples are [first_j, last_j] of t[] and y[]; grad is
// [L * (P + 1)]; loss accumulates L.
__global__ void __launch_bounds__(LM_TRAIN_THREADS) k_lm_grad(const float* __restrict__ t, const float* __restrict__ y,
                                                              size_t m, LmTables T, float* __restrict__ grad,
                                                              double* __restrict__ loss) {
    __shared__ float bp[LM_P - 1], pv[LM_P + 1];
    __shared__ float g_red[(LM_TRAIN_THREADS / 32) * (LM_P + 1)], e_red[(LM_TRAIN_THREADS / 32) * 2];
    const int j = blockIdx.x;
    const int f = T.first[j], l = T.last[j];
    if (f < 0 || l < f || (size_t)l >= m) return;  // empty leaf (or a range outside the samples)
    if (threadIdx.x < LM_P - 1) bp[threadIdx.x] = T.bp[(size_t)j * (LM_P - 1) + threadIdx.x];
    if (threadIdx.x <= LM_P) pv[threadIdx.x] = T.v[(size_t)j * (LM_P + 1) + threadIdx.x];
    __syncthreads();
    float g[LM_P + 1];
    float sse = 0.f, emax = 0.f;
    lm_leaf_grads(
        f, l, bp, pv, T.y0[j], T.h[j], 1.f / (float)m, [&](int i) { return t[i]; }, [&](int i) { return y[i]; },
        g_red, e_red, g, sse, emax);
    if (threadIdx.x == 0) {
        for (int q = 0; q <= LM_P; ++q) grad[(size_t)j * (LM_P + 1) + q] = g[q];
        atomicAdd(loss, (double)sse / (double)m);
    }
}

// Test hook: overwrite the trained heights and leaf ranks with arbitrary
// values (NaN, +-1e30, random) to show that the bounds keep the map monotone.
__global__ void k_lm_corrupt(int leaves, LmTables T, unsigned long long seed) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < leaves; j += gridDim.x * blockDim.x) {
        unsigned long long z = seed + 0x9e3779b97f4a7c15ull * (unsigned long long)(j + 1);
        for (int q = 0; q < LM_P + 3; ++q) {
            z ^= z << 13;
            z ^= z >> 7;
            z ^= z << 17;
            const unsigned int r = (unsigned int)(z >> 32);
            const int kind = r & 7;
            const float val = kind == 0   ? __int_as_float(0x7fc00000)
                              : kind == 1 ? -1e30f
                              : kind == 2 ? 1e30f
                                          : ((float)(r >> 8) / 8388608.f - 1.f) * 4.f;
            if (q <= LM_P) T.v[(size_t)j * (LM_P + 1) + q] = val;
            else if (q == LM_P + 1) T.y0[j] = val;
            else T.h[j] = val;
        }
    }
}

// Bucket-space heights and per-leaf bucket ranges. Every value is sanitised
// (NaN dropped, clamped, running maxima) so the map is non-decreasing whatever
// the fit produced: breakpoints and heights non-decreasing within a leaf, and
// lo_j >= hi_{j-1}. One CTA of 1024 threads, two leaves a thread.
__global__ void __launch_bounds__(1024) k_lm_bounds(int leaves, int buckets, LmTables T) {
    __shared__ int wmax[32];
    const float B = (float)buckets;
    int a[2] = {0, 0}, b[2] = {0, 0};
    for (int e = 0; e < 2; ++e) {
        const int j = threadIdx.x * 2 + e;
        if (j >= leaves) break;
        float y0 = T.y0[j], h = T.h[j];
        if (!(y0 == y0) || !(h == h)) y0 = h = 0.f;  // NaN
        y0 = fminf(fmaxf(y0, 0.f), 1.f);
        h = fminf(fmaxf(h, 0.f), 1.f);
        float* bp = T.bp + (size_t)j * (LM_P - 1);
        float prev = 0.f;
        for (int q = 0; q < LM_P - 1; ++q) {
            prev = fmaxf(prev, fminf(bp[q], 1.f));  // fmaxf drops a NaN
            bp[q] = prev;
        }
        const float* v = T.v + (size_t)j * (LM_P + 1);
        float* c = T.c + (size_t)j * (LM_P + 1);
        float pv = 0.f, pc = 0.f;
        for (int q = 0; q <= LM_P; ++q) {
            pv = fmaxf(pv, fminf(v[q], 1.f));
            pc = fmaxf(pc, fminf(fmaf(h, pv, y0) * B, B));
            c[q] = pc;
        }
        a[e] = min((int)c[0], buckets - 1);
        b[e] = max(a[e], min((int)c[LM_P], buckets - 1));
        if (T.first[j] < 0) a[e] = b[e] = 0;  // no sample and no key: any range will do
    }
    // inclusive max-scan of b over the leaves: hi_j; lo_j = max(a_j, hi_{j-1})
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = max(b[0], b[1]);
    for (int o = 1; o < 32; o <<= 1) {
        const int yv = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x = max(x, yv);
    }
    if (lane == 31) wmax[warp] = x;
    __syncthreads();
    int run = 0;
    for (int w = 0; w < warp; ++w) run = max(run, wmax[w]);
    const int prev_lane = __shfl_up_sync(0xffffffffu, x, 1);
    if (lane > 0) run = max(run, prev_lane);
    for (int e = 0; e < 2; ++e) {
        const int j = threadIdx.x * 2 + e;
        if (j >= leaves) break;
        const int lo = max(a[e], run);
        const int hi = max(lo, b[e]);
        LmLeaf lf = T.leaf[j];
        lf.lo = (short)lo;
        lf.hi = (short)hi;
        T.leaf[j] = lf;
        run = hi;
    }
}


// ---- partition ---------------------------------------------------------------
// Shared-memory copy of a fitted model for the count kernel.
__host__ __device__ inline size_t lm_smem_bytes(int leaves) {
    return (size_t)leaves * sizeof(LmLeaf) + (size_t)(1 << lm_depth(leaves)) * 4 + (size_t)leaves * (LM_P - 1) * 4 +
           (size_t)leaves * (LM_P + 1) * 4 + 64;
}

struct LmView {
    const LmLeaf* leaf;
    const uint32_t* rootk;
    const float* bp;
    const float* c;
};

__device__ __forceinline__ LmView lm_load(unsigned char* sm, int L, const LmTables& T) {
    const int nE = 1 << lm_depth(L);
    LmLeaf* leaf = reinterpret_cast<LmLeaf*>(sm);
    uint32_t* rootk = reinterpret_cast<uint32_t*>(leaf + L);
    float* bp = reinterpret_cast<float*>(rootk + nE);
    float* c = bp + (size_t)L * (LM_P - 1);
    for (int j = threadIdx.x; j < L; j += blockDim.x) leaf[j] = T.leaf[j];
    for (int j = threadIdx.x; j < nE; j += blockDim.x) rootk[j] = T.rootk[j];
    for (int j = threadIdx.x; j < L * (LM_P - 1); j += blockDim.x) bp[j] = T.bp[j];
    for (int j = threadIdx.x; j < L * (LM_P + 1); j += blockDim.x) c[j] = T.c[j];
    return LmView{leaf, rootk, bp, c};
}

// Bucket of a key in leaf j (the root search already done): the leaf's
// piecewise-linear CDF, clamped into the piece's and the leaf's bucket range.
template <typename U>
__device__ __forceinline__ int lm_leaf_bucket(const LmView& V, int j, U key) {
    const LmLeaf lf = V.leaf[j];
    const float t = lm_t(key, lf.klo, lf.winv);
    int k;
    float frac;
    lm_piece(V.bp + (size_t)j * (LM_P - 1), t, k, frac);
    const float* c = V.c + (size_t)j * (LM_P + 1);
    const float c0 = c[k], c1 = c[k + 1];
    const int b = (int)fmaf(c1 - c0, frac, c0);
    return min(max(min(max(b, (int)c0), (int)c1), (int)lf.lo), (int)lf.hi);
}

// Buckets of N keys at once. The root searches run level by level over all
// N keys, so each level's N shared reads are independent and overlap (one
// key's search alone is a chain of `depth` dependent reads).
template <typename U, int N>
__device__ __forceinline__ void lm_buckets(const LmHead& hd, const LmView& V, int depth, const U (&key)[N],
                                           int (&b)[N]) {
    if (!hd.use_model) {
#pragma unroll
        for (int e = 0; e < N; ++e) {
            const unsigned long long k = (unsigned long long)key[e];
            const float x = k <= hd.kmin ? 0.f : k >= hd.kmax ? 1.f : __ull2float_rn(k - hd.kmin) * hd.inv_range;
            b[e] = min(hd.buckets - 1, (int)(x * (float)hd.buckets));
        }
        return;
    }
    uint32_t p[N];
    int node[N];
#pragma unroll
    for (int e = 0; e < N; ++e) {
        p[e] = lm_prefix(hd, key[e]);
        node[e] = 1;
    }
    for (int s = 0; s < depth; ++s) {
#pragma unroll
        for (int e = 0; e < N; ++e) node[e] = 2 * node[e] + (V.rootk[node[e]] <= p[e] ? 1 : 0);
    }
#pragma unroll
    for (int e = 0; e < N; ++e) b[e] = lm_leaf_bucket<U>(V, min(node[e] - (1 << depth), hd.leaves - 1), key[e]);
}

constexpr int LM_ILP = 4;

// Every key's bucket to ids[], and the bucket sizes (added into totals[]).
template <typename U, int XF>
__global__ void __launch_bounds__(1024) k_lm_count(const U* __restrict__ src, size_t n, const LmHead* __restrict__ head,
                                                   LmTables T, unsigned short* __restrict__ ids,
                                                   unsigned long long* __restrict__ totals) {
    extern __shared__ __align__(16) unsigned char lsm[];
    const LmHead hd = *head;
    const LmView V = lm_load(lsm, hd.leaves, T);
    unsigned int* hist = reinterpret_cast<unsigned int*>(lsm + lm_smem_bytes(hd.leaves));
    for (int b = threadIdx.x; b < hd.buckets; b += blockDim.x) hist[b] = 0;
    __syncthreads();
    const int depth = lm_depth(hd.leaves);
    const size_t step = (size_t)gridDim.x * blockDim.x * LM_ILP;
    for (size_t base = (size_t)blockIdx.x * blockDim.x * LM_ILP + threadIdx.x; base < n; base += step) {
        U k[LM_ILP];
#pragma unroll
        for (int e = 0; e < LM_ILP; ++e) {
            const size_t i = base + (size_t)e * blockDim.x;
            k[e] = i < n ? src[i] : (U)0;
        }
        U key[LM_ILP];
#pragma unroll
        for (int e = 0; e < LM_ILP; ++e) key[e] = to_key<U, XF>(k[e]);
        int bk[LM_ILP];
        lm_buckets<U, LM_ILP>(hd, V, depth, key, bk);
#pragma unroll
        for (int e = 0; e < LM_ILP; ++e) {
            const size_t i = base + (size_t)e * blockDim.x;
            if (i < n) {
                ids[i] = (unsigned short)bk[e];
                atomicAdd(&hist[bk[e]], 1u);
            }
        }
    }
    __syncthreads();
    for (int b = threadIdx.x; b < hd.buckets; b += blockDim.x)
        if (hist[b]) atomicAdd(&totals[b], (unsigned long long)hist[b]);
}

constexpr int LM_SUPERS = 128;        // first scatter sweep: 128 groups of consecutive buckets
constexpr int LM_SPLIT_IPT = 8;
constexpr int LM_SPLIT_THREADS = 512;  // two CTAs an SM: one's barriers and loads overlap the other's work
constexpr int LM_SPLIT_TILE = LM_SPLIT_THREADS * LM_SPLIT_IPT;

// Exclusive scan of the bucket sizes into offsets[0..B], the largest bucket,
// the scatter cursors (cur2[b] = offsets[b], cur1[S] = offsets[S * B/128]),
// and tiles_before[S]: the second sweep's tiles in groups before S.
__global__ void __launch_bounds__(1024) k_lm_bucket_scan(const unsigned long long* __restrict__ totals, int buckets,
                                                         unsigned long long* __restrict__ offsets,
                                                         unsigned long long* __restrict__ max_bucket,
                                                         unsigned long long* __restrict__ cur1,
                                                         unsigned long long* __restrict__ cur2,
                                                         unsigned int* __restrict__ tiles_before) {
    __shared__ unsigned long long warp_sum[32];
    __shared__ unsigned long long carry;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) carry = 0;
    unsigned long long mx = 0;
    __syncthreads();
    for (int base = 0; base < buckets; base += 1024) {
        const int b = base + threadIdx.x;
        const unsigned long long v = b < buckets ? totals[b] : 0ull;
        mx = v > mx ? v : mx;
        unsigned long long x = v;
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long yy = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += yy;
        }
        if (lane == 31) warp_sum[warp] = x;
        __syncthreads();
        unsigned long long before = carry;
        for (int w = 0; w < warp; ++w) before += warp_sum[w];
        if (b < buckets) {
            offsets[b] = before + x - v;
            cur2[b] = before + x - v;
        }
        __syncthreads();
        if (threadIdx.x == 1023) carry = before + x;
        __syncthreads();
    }
    if (threadIdx.x == 0) offsets[buckets] = carry;
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long yy = __shfl_xor_sync(0xffffffffu, mx, o);
        mx = yy > mx ? yy : mx;
    }
    if (lane == 0) atomicMax(max_bucket, mx);
    __syncthreads();  // offsets[] written by this block are visible to it now
    if (threadIdx.x < 32) {
        const int per = buckets / LM_SUPERS;
        unsigned int run = 0;
        for (int g = 0; g < LM_SUPERS / 32; ++g) {
            const int S = g * 32 + lane;
            const unsigned long long lo = offsets[S * per], hi = offsets[(S + 1) * per];
            cur1[S] = lo;
            const unsigned int t = (unsigned int)((hi - lo + LM_SPLIT_TILE - 1) / LM_SPLIT_TILE);
            unsigned int x = t;
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned int yy = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += yy;
            }
            tiles_before[S] = run + x - t;
            run += __shfl_sync(0xffffffffu, x, 31);
        }
        if (lane == 0) tiles_before[LM_SUPERS] = run;
    }
}

// Shared memory of a scatter sweep: the staged tile as it arrives (keys and
// bucket ids, each with 32 bytes of room: a copy widened to 16-byte bounds
// at both ends adds at most 15 + 15 bytes), the tile grouped by digit,
// per-digit counts, starts, reserved global bases and range ends, and the
// staging barrier.
template <typename U>
struct LmSplitSmem {
    static constexpr size_t al(size_t x) { return (x + 15) / 16 * 16; }
    static constexpr size_t stage_k = 0;
    static constexpr size_t stage_i = al(stage_k + (size_t)LM_SPLIT_TILE * sizeof(U) + 32);
    static constexpr size_t keys = al(stage_i + (size_t)LM_SPLIT_TILE * 2 + 32);
    static constexpr size_t ids = keys + (size_t)LM_SPLIT_TILE * sizeof(U);
    static constexpr size_t cnt = al(ids + (size_t)LM_SPLIT_TILE * 2);
    static constexpr size_t start = cnt + 256 * 4;
    static constexpr size_t gbase = start + 256 * 4;
    static constexpr size_t gend = gbase + 256 * 8;
    static constexpr size_t bar = gend + 256 * 8;
    static constexpr size_t bytes = bar + 64;
};

// One scatter tile: `len` keys and ids (staged in shared memory), grouped by
// digit = (id >> shift) & (bins - 1), each digit's run written at a range of
// dst reserved with one atomic on cur[digit] (the order inside a bucket is
// free: the buckets are sorted afterwards), so the stores are coalesced runs.
// Digit d's range of dst ends at ends[(d + 1) * end_stride]; a store past it
// (counts that disagree with the ids) is dropped and flagged. `staged` runs
// (on every thread) once the staging area has been read, so the next tile
// can start arriving there.
template <typename U, bool WRITE_IDS, typename Staged>
__device__ __forceinline__ void lm_split_tile(const U* src, const unsigned short* ids, int len, int shift, int bins,
                                              unsigned long long* __restrict__ cur,
                                              const unsigned long long* __restrict__ ends, int end_stride,
                                              U* __restrict__ dst, unsigned short* __restrict__ dst_ids,
                                              unsigned char* sm, uint32_t* __restrict__ error, Staged staged) {
    U* sk = reinterpret_cast<U*>(sm + LmSplitSmem<U>::keys);
    unsigned short* sid = reinterpret_cast<unsigned short*>(sm + LmSplitSmem<U>::ids);
    unsigned int* cnt = reinterpret_cast<unsigned int*>(sm + LmSplitSmem<U>::cnt);
    unsigned int* start = reinterpret_cast<unsigned int*>(sm + LmSplitSmem<U>::start);
    unsigned long long* gbase = reinterpret_cast<unsigned long long*>(sm + LmSplitSmem<U>::gbase);
    unsigned long long* gend = reinterpret_cast<unsigned long long*>(sm + LmSplitSmem<U>::gend);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid < 256) cnt[tid] = 0;
    __syncthreads();
    U k[LM_SPLIT_IPT];
    unsigned short id[LM_SPLIT_IPT];
    int slot[LM_SPLIT_IPT];
#pragma unroll
    for (int e = 0; e < LM_SPLIT_IPT; ++e) {
        const int i = e * LM_SPLIT_THREADS + tid;
        if (i < len) {
            k[e] = src[i];
            id[e] = ids[i];
            slot[e] = (int)atomicAdd(&cnt[(id[e] >> shift) & (bins - 1)], 1u);
        }
    }
    __syncthreads();
    staged();
    if (warp < 8) {  // exclusive scan of cnt[0..256), one warp a 32-digit slice, then across slices
        const int d = warp * 32 + lane;
        const unsigned int v = d < bins ? cnt[d] : 0u;
        unsigned int x = v;
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned int yy = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += yy;
        }
        start[d] = x - v;
        if (lane == 31) reinterpret_cast<unsigned int*>(gbase)[warp] = x;  // slice totals, scratch
    }
    __syncthreads();
    if (tid < 256) {
        unsigned int before = 0;
        for (int w = 0; w < (tid >> 5); ++w) before += reinterpret_cast<unsigned int*>(gbase)[w];
        start[tid] += before;
    }
    __syncthreads();
    if (tid < bins) {
        gbase[tid] = cnt[tid] ? atomicAdd(&cur[tid], (unsigned long long)cnt[tid]) : 0ull;
        gend[tid] = ends[(size_t)(tid + 1) * end_stride];
    }
#pragma unroll
    for (int e = 0; e < LM_SPLIT_IPT; ++e) {
        const int i = e * LM_SPLIT_THREADS + tid;
        if (i < len) {
            const int p = (int)start[(id[e] >> shift) & (bins - 1)] + slot[e];
            sk[p] = k[e];
            sid[p] = id[e];
        }
    }
    __syncthreads();
    for (int i = tid; i < len; i += LM_SPLIT_THREADS) {
        const int d = (sid[i] >> shift) & (bins - 1);
        const unsigned long long g = gbase[d] + (unsigned long long)(i - (int)start[d]);
        if (g < gend[d]) {
            dst[g] = sk[i];
            if (WRITE_IDS) dst_ids[g] = sid[i];
        } else {
            atomicOr(error, ERR_BOUNDS);
        }
    }
    __syncthreads();
}

// A persistent sweep's staging: bulk copies (no multicast) of a tile's keys
// and ids into shared memory, completing on one mbarrier. A tile that starts
// off a 16-byte boundary is copied from the boundary below (and up to the
// boundary above its end: neither crosses a page), and read from `pre`
// elements in.
template <typename U>
struct LmStage {
    unsigned char* sm;
    uint64_t* bar;
    uint32_t parity;
    __device__ static int pre_k(const U* p) { return (int)(((uintptr_t)p & 15) / sizeof(U)); }
    __device__ static int pre_i(const unsigned short* p) { return (int)(((uintptr_t)p & 15) / 2); }
    // thread 0: start the copy of [k, k + len) and [i, i + len)
    __device__ void issue(const U* k, const unsigned short* i, int len) {
        if (len <= 0) {
            mbar_arrive_expect_tx(bar, 0);
            return;
        }
        const uintptr_t ka = (uintptr_t)k & ~(uintptr_t)15, kz = ((uintptr_t)(k + len) + 15) & ~(uintptr_t)15;
        const uintptr_t ia = (uintptr_t)i & ~(uintptr_t)15, iz = ((uintptr_t)(i + len) + 15) & ~(uintptr_t)15;
        fence_proxy_async_smem();
        mbar_arrive_expect_tx(bar, (uint32_t)((kz - ka) + (iz - ia)));
        bulk_g2s(sm + LmSplitSmem<U>::stage_k, (const void*)ka, (uint32_t)(kz - ka), bar);
        bulk_g2s(sm + LmSplitSmem<U>::stage_i, (const void*)ia, (uint32_t)(iz - ia), bar);
    }
    // every thread: wait for the copy (bounded; a timeout is flagged and the
    // tile's writes stay inside their ranges)
    __device__ void wait(uint32_t* error) {
        if (!mbar_wait(bar, parity)) atomicOr(error, ERR_TIMEOUT);
        parity ^= 1u;
    }
};

// First sweep: keys (and ids) into LM_SUPERS groups of consecutive buckets.
// Persistent CTAs take every gridDim.x-th tile; the next tile's copy into
// shared memory starts as soon as this tile's keys are in registers.
template <typename U>
__global__ void __launch_bounds__(LM_SPLIT_THREADS, 2) k_lm_split1(const U* __restrict__ src, const unsigned short* __restrict__ ids,
                                                       size_t n, int shift, unsigned long long* __restrict__ cur1,
                                                       const unsigned long long* __restrict__ offsets,
                                                       U* __restrict__ dst, unsigned short* __restrict__ dst_ids,
                                                       uint32_t* __restrict__ error) {
    extern __shared__ __align__(128) unsigned char ssm[];
    const size_t tiles = (n + LM_SPLIT_TILE - 1) / LM_SPLIT_TILE;
    LmStage<U> st{ssm, reinterpret_cast<uint64_t*>(ssm + LmSplitSmem<U>::bar), 0u};
    auto span = [&](size_t tile, size_t& t0, int& len) {
        t0 = tile * LM_SPLIT_TILE;
        len = (int)min((size_t)LM_SPLIT_TILE, n - t0);
    };
    if (threadIdx.x == 0) {
        mbar_init(st.bar, 1);
        fence_mbar_init();
        if (blockIdx.x < tiles) {
            size_t t0;
            int len;
            span(blockIdx.x, t0, len);
            st.issue(src + t0, ids + t0, len);
        }
    }
    __syncthreads();
    for (size_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        size_t t0;
        int len;
        span(tile, t0, len);
        st.wait(error);
        const U* sk = reinterpret_cast<const U*>(ssm + LmSplitSmem<U>::stage_k) + LmStage<U>::pre_k(src + t0);
        const unsigned short* si =
            reinterpret_cast<const unsigned short*>(ssm + LmSplitSmem<U>::stage_i) + LmStage<U>::pre_i(ids + t0);
        lm_split_tile<U, true>(sk, si, len, shift, LM_SUPERS, cur1, offsets, 1 << shift, dst, dst_ids, ssm, error, [&] {
            if (threadIdx.x == 0 && tile + gridDim.x < tiles) {
                size_t u0;
                int ulen;
                span(tile + gridDim.x, u0, ulen);
                st.issue(src + u0, ids + u0, ulen);
            }
        });
    }
}

// The second sweep's tile number `tile` as (group S, start, length); tiles
// never cross a group's boundary (tiles_before[] numbers them group by group).
__device__ __forceinline__ int lm_tile2(unsigned int tile, int per, const unsigned long long* __restrict__ offsets,
                                        const unsigned int* __restrict__ tiles_before, unsigned long long& t0,
                                        int& len) {
    int lo = 0, hi = LM_SUPERS - 1;  // the group S with tiles_before[S] <= tile < tiles_before[S + 1]
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (tiles_before[mid] <= tile) lo = mid;
        else hi = mid - 1;
    }
    const unsigned long long g0 = offsets[lo * per], g1 = offsets[(lo + 1) * per];
    t0 = g0 + (unsigned long long)(tile - tiles_before[lo]) * LM_SPLIT_TILE;
    len = t0 < g1 ? (int)min((unsigned long long)LM_SPLIT_TILE, g1 - t0) : 0;
    return lo;
}

// Second sweep: inside each group, keys to their buckets; persistent CTAs
// with the next tile's copy started early, as in the first sweep.
template <typename U>
__global__ void __launch_bounds__(LM_SPLIT_THREADS, 2) k_lm_split2(const U* __restrict__ src, const unsigned short* __restrict__ ids,
                                                       int buckets, const unsigned long long* __restrict__ offsets,
                                                       const unsigned int* __restrict__ tiles_before,
                                                       unsigned long long* __restrict__ cur2, U* __restrict__ dst,
                                                       uint32_t* __restrict__ error) {
    extern __shared__ __align__(128) unsigned char ssm[];
    const unsigned int tiles = tiles_before[LM_SUPERS];
    const int per = buckets / LM_SUPERS;
    LmStage<U> st{ssm, reinterpret_cast<uint64_t*>(ssm + LmSplitSmem<U>::bar), 0u};
    if (threadIdx.x == 0) {
        mbar_init(st.bar, 1);
        fence_mbar_init();
        if (blockIdx.x < tiles) {
            unsigned long long t0;
            int len;
            lm_tile2(blockIdx.x, per, offsets, tiles_before, t0, len);
            st.issue(src + t0, ids + t0, len);
        }
    }
    __syncthreads();
    for (unsigned int tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        unsigned long long t0;
        int len;
        const int S = lm_tile2(tile, per, offsets, tiles_before, t0, len);
        st.wait(error);
        const U* sk = reinterpret_cast<const U*>(ssm + LmSplitSmem<U>::stage_k) + LmStage<U>::pre_k(src + t0);
        const unsigned short* si =
            reinterpret_cast<const unsigned short*>(ssm + LmSplitSmem<U>::stage_i) + LmStage<U>::pre_i(ids + t0);
        lm_split_tile<U, false>(sk, si, len, 0, per, cur2 + (size_t)S * per, offsets + (size_t)S * per, 1, dst, nullptr,
                                ssm, error, [&] {
                                    if (threadIdx.x == 0 && tile + gridDim.x < tiles) {
                                        unsigned long long u0;
                                        int ulen;
                                        lm_tile2(tile + gridDim.x, per, offsets, tiles_before, u0, ulen);
                                        st.issue(src + u0, ids + u0, ulen);
                                    }
                                });
    }
}

// ---- bucket finish -----------------------------------------------------------
// Every bucket sorted from `in` (the partition) into `out`, one CTA a bucket
// at a time, by the segmented sort's MSD routine (msd_sort: one digit pass
// over the bucket's key range in shared memory, the CTA-level LSD for
// buckets above its capacity). The next bucket is claimed early and brought
// into L2 while this one is sorted.
template <typename U, int XF>
__global__ void __launch_bounds__(1024, 1) k_lm_finish(const U* __restrict__ in, U* __restrict__ out,
                                                       U* __restrict__ scratch,
                                                       const unsigned long long* __restrict__ offsets, int buckets,
                                                       unsigned int* __restrict__ counter) {
    extern __shared__ __align__(16) unsigned char fsm[];
    int* item_s = reinterpret_cast<int*>(fsm + MsdSmem<U>::misc) + 48;
    const int tid = threadIdx.x;
    if (tid == 0) item_s[1] = (int)atomicAdd(counter, 1u);
    for (;;) {
        if (tid == 0) {
            item_s[0] = item_s[1];
            const int nb = (int)atomicAdd(counter, 1u);
            item_s[1] = nb;
            if (nb < buckets) prefetch_l2(in + offsets[nb], in + min(offsets[nb + 1], offsets[nb] + (1ull << 22)));
        }
        __syncthreads();
        const int b = item_s[0];
        __syncthreads();
        if (b >= buckets) break;
        const unsigned long long lo = offsets[b];
        msd_sort<U, XF>(in + lo, out + lo, scratch + lo, (int)(offsets[b + 1] - lo), fsm);
    }
}

}  // namespace ts
