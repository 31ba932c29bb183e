// ts_pipeline.cuh — the host-slice sort with its copies overlapped.
//
// The crate's sort takes a host slice (src/lib.rs:99); on the device the
// copies in and out cost far more than the sort (PCIe moves ~55 GB/s each
// way, the sort ~250 GB/s of keys). With the copies serialised the call
// costs copy-in + sort + copy-out. Here the slice crosses as C chunks on a
// second stream; chunk i is sorted (the plain LSD, in place, with the
// partner buffer's range of the chunk as scratch) while chunk i + 1 is
// still in flight, and equal-sized sorted runs are merged pairwise as soon
// as both exist (a binary counter of runs, so merges of early chunks also
// overlap later copies). The last merge runs in output slices; each slice
// is copied out while the next one is merged. The call then costs about
// copy-in + (sort of one chunk + the last merges' first slice) + copy-out.
//
// Buffers: chunks arrive in `keys` (X); a run at merge level L lives in X
// for even L and in `alt` (Y) for odd L, over its own index range, so the
// scratch a chunk sort takes (Y over the chunk's range) and the target of
// every merge never overlap a live run. Host calls are ordered so that the
// copy of chunk i + 2 is issued after the sort of chunk i and every copy out
// after the last merge.
//
// The same chunks and merge tree (run_pipeline) serve sort_by_key's order()
// (pipeline_order): a chunk's run is its stable order, and runs of positions
// are merged by the keys they point to. Pageable host slices cross through
// pinned staging slots (ts_transfer.h).
#pragma once

#include <algorithm>
#include <vector>

#include "ts_engine.cuh"
#include "ts_merge.cuh"
#include "ts_transfer.h"

namespace ts {

// One merge of `total` outputs on the context's stream: splits(grid,
// tiles) launches the split search, tiles(grid, t0, t1) a range of output
// tiles. When `sliced` the tiles go in PIPE_SLICES output slices; slice p
// ends at output slice_end[p] and its completion is recorded in slice_ev[p].
template <typename Splits, typename Tiles>
ts_status enqueue_merge_launches(ts_ctx* c, size_t total, bool sliced, cudaEvent_t* slice_ev, size_t* slice_end,
                                 Splits splits, Tiles tiles_fn) {
    const size_t tiles = (total + MERGE_TILE - 1) / MERGE_TILE;
    const int sg = (int)std::min<size_t>((tiles + 1 + 255) / 256, (size_t)c->sm_count * 8);
    splits(std::max(sg, 1), tiles);
    ++c->launches;
    const int parts = sliced ? PIPE_SLICES : 1;
    for (int p = 0; p < parts; ++p) {
        const size_t t0 = tiles * p / parts, t1 = tiles * (p + 1) / parts;
        if (t1 > t0) {
            tiles_fn((int)std::min<size_t>(t1 - t0, (size_t)c->sm_count * 8), t0, t1);
            ++c->launches;
        }
        if (sliced) {
            slice_end[p] = std::min(total, t1 * (size_t)MERGE_TILE);
            TS_CUDA(c, cudaEventRecord(slice_ev[p], c->stream));
        }
    }
    TS_CUDA(c, cudaGetLastError());
    return TS_OK;
}

// Merge sorted key runs a and b into out.
template <typename U, int XF>
ts_status enqueue_merge(ts_ctx* c, const U* a, size_t na, const U* b, size_t nb, U* out, bool sliced,
                        cudaEvent_t* slice_ev, size_t* slice_end) {
    size_t* split = (size_t*)c->pipe.p;
    return enqueue_merge_launches(
        c, na + nb, sliced, slice_ev, slice_end,
        [&](int g, size_t tiles) { k_merge_splits<U, XF><<<g, 256, 0, c->stream>>>(a, na, b, nb, tiles, split); },
        [&](int g, size_t t0, size_t t1) {
            k_merge_tiles<U, XF><<<g, MERGE_THREADS, 0, c->stream>>>(a, na, b, nb, out, split, t0, t1);
        });
}

// Merge position runs a (+ a_base) and b (+ b_base) of `keys` into out.
template <typename U, int XF>
ts_status enqueue_merge_pos(ts_ctx* c, const U* keys, const uint32_t* a, size_t na, uint32_t a_base,
                            const uint32_t* b, size_t nb, uint32_t b_base, uint32_t* out, bool sliced,
                            cudaEvent_t* slice_ev, size_t* slice_end) {
    size_t* split = (size_t*)c->pipe.p;
    return enqueue_merge_launches(
        c, na + nb, sliced, slice_ev, slice_end,
        [&](int g, size_t tiles) {
            k_merge_pos_splits<U, XF><<<g, 256, 0, c->stream>>>(keys, a, na, a_base, b, nb, b_base, tiles, split);
        },
        [&](int g, size_t t0, size_t t1) {
            k_merge_pos_tiles<U, XF><<<g, MERGE_THREADS, 0, c->stream>>>(keys, a, na, a_base, b, nb, b_base, out,
                                                                         split, t0, t1);
        });
}

// The chunks, the merge tree over their sorted runs, and the copies of one
// pipelined call. sort_chunk(i, b, e) enqueues chunk i's sort (into its
// level-0 run); merge(L, r1, r2, last) enqueues the merge of two level-L
// runs. The copy in of chunk i + 2 is issued after chunk i's sort, so a
// pageable slice, whose staged copies hold this thread, overlaps the work
// already queued.
template <typename CopyIn, typename SortChunk, typename Merge>
ts_status run_pipeline(ts_ctx* c, size_t n, CopyIn copy_chunk, SortChunk sort_chunk, Merge merge) {
    const int C = c->transfer_chunks;
    const size_t chunk = ((n + C - 1) / C + 255) / 256 * 256;  // chunk starts 256 elements apart: 16-byte aligned
    auto lo = [&](int i) { return std::min(n, (size_t)i * chunk); };
    cudaEvent_t* in_ev = c->pipe_events.data();  // [C] chunk i is on the device
    ts_status s;
    // the copies start behind whatever the context's stream already holds
    cudaEvent_t ready_ev = in_ev[C + PIPE_SLICES];
    TS_CUDA(c, cudaEventRecord(ready_ev, c->stream));
    TS_CUDA(c, cudaStreamWaitEvent(c->copy_stream, ready_ev, 0));
    auto copy_in = [&](int i) -> ts_status {
        if (i >= C) return TS_OK;
        ts_status st = copy_chunk(lo(i), lo(i + 1));
        if (st != TS_OK) return st;
        TS_CUDA(c, cudaEventRecord(in_ev[i], c->copy_stream));
        return TS_OK;
    };
    mark(c, "pipeline");
    if ((s = copy_in(0)) != TS_OK) return s;
    if ((s = copy_in(1)) != TS_OK) return s;
    struct Run {
        size_t b, e;
        int level;
    };
    std::vector<Run> runs;
    for (int i = 0; i < C; ++i) {
        TS_CUDA(c, cudaStreamWaitEvent(c->stream, in_ev[i], 0));
        if ((s = sort_chunk(lo(i), lo(i + 1))) != TS_OK) return s;
        runs.push_back({lo(i), lo(i + 1), 0});
        while (runs.size() >= 2 && runs[runs.size() - 1].level == runs[runs.size() - 2].level) {
            const Run r2 = runs.back();
            runs.pop_back();
            const Run r1 = runs.back();
            runs.pop_back();
            mark(c, "merge");
            if ((s = merge(r1.level, r1.b, r1.e, r2.e, i == C - 1 && runs.empty())) != TS_OK) return s;
            runs.push_back({r1.b, r2.e, r1.level + 1});
        }
        if ((s = copy_in(i + 2)) != TS_OK) return s;
    }
    mark(c, "end");
    return TS_OK;
}

// Enqueue the sort of the host slice h[0, n) with the copies overlapped
// (c->transfer_chunks a power of two, at least 2); the context's stream ends
// behind the last copy out.
template <typename U, int XF>
ts_status pipeline_body(ts_ctx* c, U* h, size_t n) {
    ts_status s;
    if ((s = grow(c, c->keys, n * sizeof(U), "keys")) != TS_OK) return s;
    if ((s = grow(c, c->alt, n * sizeof(U), "scratch keys")) != TS_OK) return s;
    if ((s = grow(c, c->pipe, ((n + MERGE_TILE - 1) / MERGE_TILE + 1) * sizeof(size_t), "merge splits")) != TS_OK)
        return s;
    if ((s = pipe_resources(c, (size_t)c->transfer_chunks + PIPE_SLICES + 2)) != TS_OK) return s;
    Transfer T(c, h);
    U* X = (U*)c->keys.p;  // chunks arrive here; even merge levels
    U* Y = (U*)c->alt.p;   // odd merge levels; a chunk sort's scratch
    size_t slice_end[PIPE_SLICES] = {};
    U* final_buf = X;
    s = run_pipeline(
        c, n, [&](size_t b, size_t e) { return T.in(X + b, h + b, (e - b) * sizeof(U)); },
        [&](size_t b, size_t e) { return sort_keys_device<U, XF>(c, X + b, e - b, Y + b); },
        [&](int L, size_t b, size_t m, size_t e, bool last) {
            U* src = (L & 1) ? Y : X;
            U* dst = (L & 1) ? X : Y;
            if (last) final_buf = dst;
            return enqueue_merge<U, XF>(c, src + b, m - b, src + m, e - m, dst + b, last, slice_events(c), slice_end);
        });
    if (s != TS_OK) return s;
    size_t end_bytes[PIPE_SLICES];
    for (int p = 0; p < PIPE_SLICES; ++p) end_bytes[p] = slice_end[p] * sizeof(U);
    if ((s = T.out(h, final_buf, end_bytes, slice_events(c), PIPE_SLICES)) != TS_OK) return s;
    TS_CUDA(c, cudaEventRecord(done_event(c), c->copy_stream));
    TS_CUDA(c, cudaStreamWaitEvent(c->stream, done_event(c), 0));
    return TS_OK;
}

// The pipelined host sort: returns once the sorted keys are back in h.
template <typename U, int XF>
ts_status pipeline_sort(ts_ctx* c, U* h, size_t n) {
    return pipeline_end(c, pipeline_body<U, XF>(c, h, n));
}

// The stable order of the host keys h_keys[0, n) (sort_by_key's order(),
// src/by_key.rs:175-233) with the copies overlapped: each chunk's keys are
// ordered by the device's stable LSD (positions within the chunk), and the
// position runs are merged by the keys they point to, which stay where they
// arrived. Enqueues it all; the context's stream ends behind the last copy
// of order[0, n) to the host.
template <typename U, int XF>
ts_status pipeline_order_body(ts_ctx* c, const U* h_keys, size_t n, uint32_t* h_order) {
    ts_status s;
    if ((s = grow(c, c->keys, n * sizeof(U), "keys")) != TS_OK) return s;
    if ((s = grow(c, c->pipe_pos[0], n * 4, "positions")) != TS_OK) return s;
    if ((s = grow(c, c->pipe_pos[1], n * 4, "positions")) != TS_OK) return s;
    if ((s = grow(c, c->pipe, ((n + MERGE_TILE - 1) / MERGE_TILE + 1) * sizeof(size_t), "merge splits")) != TS_OK)
        return s;
    if ((s = pipe_resources(c, (size_t)c->transfer_chunks + PIPE_SLICES + 2)) != TS_OK) return s;
    Transfer Tin(c, h_keys), Tout(c, h_order);  // the two share the staging slots, in stream order
    U* X = (U*)c->keys.p;
    uint32_t* P[2] = {(uint32_t*)c->pipe_pos[0].p, (uint32_t*)c->pipe_pos[1].p};
    size_t slice_end[PIPE_SLICES] = {};
    uint32_t* final_buf = P[0];
    s = run_pipeline(
        c, n, [&](size_t b, size_t e) { return Tin.in(X + b, h_keys + b, (e - b) * sizeof(U)); },
        [&](size_t b, size_t e) -> ts_status {
            if (e - b == 1) {
                TS_CUDA(c, cudaMemsetAsync(P[0] + b, 0, 4, c->stream));
                return TS_OK;
            }
            return order_device<U, XF>(c, X + b, e - b, P[0] + b);
        },
        [&](int L, size_t b, size_t m, size_t e, bool last) {
            uint32_t* src = P[L & 1];
            uint32_t* dst = P[(L + 1) & 1];
            if (last) final_buf = dst;
            // level-0 runs hold positions within their chunk
            const uint32_t ab = L == 0 ? (uint32_t)b : 0u, bb = L == 0 ? (uint32_t)m : 0u;
            return enqueue_merge_pos<U, XF>(c, X, src + b, m - b, ab, src + m, e - m, bb, dst + b, last,
                                            slice_events(c), slice_end);
        });
    if (s != TS_OK) return s;
    size_t end_bytes[PIPE_SLICES];
    for (int p = 0; p < PIPE_SLICES; ++p) end_bytes[p] = slice_end[p] * 4;
    if ((s = Tout.out(h_order, final_buf, end_bytes, slice_events(c), PIPE_SLICES)) != TS_OK) return s;
    TS_CUDA(c, cudaEventRecord(done_event(c), c->copy_stream));
    TS_CUDA(c, cudaStreamWaitEvent(c->stream, done_event(c), 0));
    return TS_OK;
}

// The pipelined host order(): returns once order[0, n) is on the host.
template <typename U, int XF>
ts_status pipeline_order(ts_ctx* c, const U* h_keys, size_t n, uint32_t* h_order) {
    return pipeline_end(c, pipeline_order_body<U, XF>(c, h_keys, n, h_order));
}

}  // namespace ts
