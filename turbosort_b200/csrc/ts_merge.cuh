// ts_merge.cuh — merging two sorted runs of keys on the device (merge path).
//
// The host-slice sort streams its input in as chunks, sorts each chunk while
// the next one is still crossing PCIe, and merges the sorted chunks pairwise;
// the last merge runs in output slices, each copied back to the host while
// the next is merged. A merge of runs a and b is two launches:
//   k_merge_splits  for every tile boundary of the output (every MERGE_TILE
//                   keys), how many of the keys before it come from a: a
//                   binary search along that output diagonal (merge path);
//   k_merge_tiles   one CTA a tile: the tile's pieces of a and b go into
//                   shared memory, each thread finds its own diagonal there,
//                   merges MERGE_IPT keys, and the tile leaves in order.
// The same two launches merge runs of positions for sort_by_key's order
// (below). Keys compare by their radix key (src/key.rs:135-197), so floats
// merge in total_cmp order. Equal radix keys are equal bit patterns, and a key-only
// merge is therefore exact whatever run an equal key is taken from; ties
// still go to a first, so the split points of neighbouring tiles agree.
#pragma once

#include "ts_common.cuh"

namespace ts {

constexpr int MERGE_THREADS = 256;
constexpr int MERGE_IPT = 8;
constexpr int MERGE_TILE = MERGE_THREADS * MERGE_IPT;  // output keys per CTA tile

// The number of a's keys among the first `diag` keys of the merge of a and b
// (a first on ties), where ka(i) and kb(j) are the radix keys of a[i] and
// b[j]. Every index it asks for lies inside a or b.
template <typename I, typename KA, typename KB>
__device__ __forceinline__ I merge_corank_by(KA ka, I na, KB kb, I nb, I diag) {
    I lo = diag > nb ? diag - nb : 0, hi = diag < na ? diag : na;
    while (lo < hi) {
        const I mid = (lo + hi) >> 1;
        if (!(kb(diag - 1 - mid) < ka(mid))) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

template <typename U, int XF, typename I>
__device__ __forceinline__ I merge_corank(const U* a, I na, const U* b, I nb, I diag) {
    return merge_corank_by<I>([&](I i) { return to_key<U, XF>(a[i]); }, na,
                              [&](I j) { return to_key<U, XF>(b[j]); }, nb, diag);
}

// split[t] for t in [0, tiles]: a's share of the first min(t * MERGE_TILE, na + nb) keys
template <typename U, int XF>
__global__ void k_merge_splits(const U* __restrict__ a, size_t na, const U* __restrict__ b, size_t nb, size_t tiles,
                               size_t* __restrict__ split) {
    const size_t total = na + nb;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t <= tiles; t += (size_t)gridDim.x * blockDim.x) {
        const size_t diag = t * (size_t)MERGE_TILE < total ? t * (size_t)MERGE_TILE : total;
        split[t] = merge_corank<U, XF, size_t>(a, na, b, nb, diag);
    }
}

// Output tiles [t_begin, t_end) of the merge of a and b into out.
template <typename U, int XF>
__global__ void __launch_bounds__(MERGE_THREADS) k_merge_tiles(const U* __restrict__ a, size_t na,
                                                               const U* __restrict__ b, size_t nb,
                                                               U* __restrict__ out, const size_t* __restrict__ split,
                                                               size_t t_begin, size_t t_end) {
    __shared__ U s[MERGE_TILE];
    const size_t total = na + nb;
    const int tid = threadIdx.x;
    for (size_t t = t_begin + blockIdx.x; t < t_end; t += gridDim.x) {
        const size_t d0 = t * (size_t)MERGE_TILE;
        const size_t d1 = d0 + MERGE_TILE < total ? d0 + MERGE_TILE : total;
        const size_t i0 = split[t], i1 = split[t + 1];
        const size_t j0 = d0 - i0;
        const int la = (int)(i1 - i0), len = (int)(d1 - d0), lb = len - la;
        // the tile's piece of a, then its piece of b
        for (int k = tid; k < len; k += MERGE_THREADS) s[k] = k < la ? a[i0 + k] : b[j0 + (k - la)];
        __syncthreads();
        const int q0 = min(len, tid * MERGE_IPT), q1 = min(len, q0 + MERGE_IPT);
        int ia = merge_corank<U, XF, int>(s, la, s + la, lb, q0);
        int ib = q0 - ia;
        U v[MERGE_IPT];
#pragma unroll
        for (int k = 0; k < MERGE_IPT; ++k) {
            if (q0 + k < q1) {
                bool take_a;
                if (ia >= la) take_a = false;
                else if (ib >= lb) take_a = true;
                else take_a = !(to_key<U, XF>(s[la + ib]) < to_key<U, XF>(s[ia]));
                v[k] = take_a ? s[ia++] : s[la + ib++];
            }
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < MERGE_IPT; ++k)
            if (q0 + k < q1) s[q0 + k] = v[k];
        __syncthreads();
        for (int k = tid; k < len; k += MERGE_THREADS) out[d0 + k] = s[k];
        __syncthreads();
    }
}

// ---- runs of positions (the stable order of sort_by_key) --------------------
// A run is a stable order of some of `keys`: positions, each plus the run's
// base (its chunk's first index while the run is one chunk's own order, 0
// once positions are global). The merge compares the keys the positions
// point to and takes a first on ties; every position of a precedes every
// position of b, so the merge of two stable orders is the stable order of
// their union, the same permutation the crate's sort_by_key gives.
template <typename U, int XF>
__global__ void k_merge_pos_splits(const U* __restrict__ keys, const uint32_t* __restrict__ a, size_t na,
                                   uint32_t a_base, const uint32_t* __restrict__ b, size_t nb, uint32_t b_base,
                                   size_t tiles, size_t* __restrict__ split) {
    const size_t total = na + nb;
    auto ka = [&](size_t i) { return to_key<U, XF>(keys[a[i] + a_base]); };
    auto kb = [&](size_t j) { return to_key<U, XF>(keys[b[j] + b_base]); };
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t <= tiles; t += (size_t)gridDim.x * blockDim.x) {
        const size_t diag = t * (size_t)MERGE_TILE < total ? t * (size_t)MERGE_TILE : total;
        split[t] = merge_corank_by<size_t>(ka, na, kb, nb, diag);
    }
}

template <typename U, int XF>
__global__ void __launch_bounds__(MERGE_THREADS) k_merge_pos_tiles(const U* __restrict__ keys,
                                                                   const uint32_t* __restrict__ a, size_t na,
                                                                   uint32_t a_base, const uint32_t* __restrict__ b,
                                                                   size_t nb, uint32_t b_base,
                                                                   uint32_t* __restrict__ out,
                                                                   const size_t* __restrict__ split, size_t t_begin,
                                                                   size_t t_end) {
    __shared__ uint32_t sp[MERGE_TILE];
    __shared__ U sk[MERGE_TILE];
    const size_t total = na + nb;
    const int tid = threadIdx.x;
    for (size_t t = t_begin + blockIdx.x; t < t_end; t += gridDim.x) {
        const size_t d0 = t * (size_t)MERGE_TILE;
        const size_t d1 = d0 + MERGE_TILE < total ? d0 + MERGE_TILE : total;
        const size_t i0 = split[t], i1 = split[t + 1];
        const size_t j0 = d0 - i0;
        const int la = (int)(i1 - i0), len = (int)(d1 - d0), lb = len - la;
        // the tile's global positions and their radix keys: a's piece, then b's
        for (int k = tid; k < len; k += MERGE_THREADS) {
            const uint32_t p = k < la ? a[i0 + k] + a_base : b[j0 + (k - la)] + b_base;
            sp[k] = p;
            sk[k] = to_key<U, XF>(keys[p]);
        }
        __syncthreads();
        const int q0 = min(len, tid * MERGE_IPT), q1 = min(len, q0 + MERGE_IPT);
        int ia = merge_corank_by<int>([&](int i) { return sk[i]; }, la, [&](int j) { return sk[la + j]; }, lb, q0);
        int ib = q0 - ia;
        uint32_t v[MERGE_IPT];
#pragma unroll
        for (int k = 0; k < MERGE_IPT; ++k) {
            if (q0 + k < q1) {
                bool take_a;
                if (ia >= la) take_a = false;
                else if (ib >= lb) take_a = true;
                else take_a = !(sk[la + ib] < sk[ia]);
                v[k] = take_a ? sp[ia++] : sp[la + ib++];
            }
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < MERGE_IPT; ++k)
            if (q0 + k < q1) sp[q0 + k] = v[k];
        __syncthreads();
        for (int k = tid; k < len; k += MERGE_THREADS) out[d0 + k] = sp[k];
        __syncthreads();
    }
}

}  // namespace ts
