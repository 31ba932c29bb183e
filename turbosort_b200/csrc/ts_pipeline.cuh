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
// A pageable host slice cannot be a DMA source or target; the driver would
// copy it through its own pinned buffer on this thread at about a quarter of
// the PCIe rate. Such a slice goes through the context's pinned staging
// slots instead: the copy pool's threads fill a slot while the DMA of the
// previous one runs, and on the way back empty a slot while the next one's
// DMA runs.
#pragma once

#include <algorithm>
#include <vector>

#include "ts_engine.cuh"
#include "ts_merge.cuh"
#include "ts_staging.h"

namespace ts {

constexpr int PIPE_SLICES = 8;                     // output slices of the last merge
constexpr int STAGE_SLOTS = 4;                     // pinned staging slots for pageable slices
constexpr size_t STAGE_SLOT_BYTES = (size_t)32 << 20;

// the pinned slots, their events and the copy threads; false if pinned
// memory cannot be had (the slice then takes the driver's own staging)
inline bool stage_resources(ts_ctx* c) {
    if (!c->stage) {
        if (cudaHostAlloc(&c->stage, STAGE_SLOTS * STAGE_SLOT_BYTES, cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            c->stage = nullptr;
            return false;
        }
    }
    while (c->stage_events.size() < (size_t)STAGE_SLOTS) {
        cudaEvent_t ev;
        if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        c->stage_events.push_back(ev);
    }
    if (!c->copy_pool) c->copy_pool = new CopyPool(copy_pool_workers());
    return true;
}

// the copy stream and the events a pipelined call uses, made once per context
inline ts_status pipe_resources(ts_ctx* c, size_t events) {
    if (!c->copy_stream) TS_CUDA(c, cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
    while (c->pipe_events.size() < events) {
        cudaEvent_t ev;
        TS_CUDA(c, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        c->pipe_events.push_back(ev);
    }
    return TS_OK;
}

// Merge sorted runs a and b into out on the context's stream. When `sliced`,
// the merge runs in PIPE_SLICES output slices; slice p ends at slice_end[p]
// and its completion is recorded in slice_ev[p].
template <typename U, int XF>
ts_status enqueue_merge(ts_ctx* c, const U* a, size_t na, const U* b, size_t nb, U* out, bool sliced,
                        cudaEvent_t* slice_ev, size_t* slice_end) {
    const size_t total = na + nb;
    const size_t tiles = (total + MERGE_TILE - 1) / MERGE_TILE;
    size_t* split = (size_t*)c->pipe.p;
    const int sg = (int)std::min<size_t>((tiles + 1 + 255) / 256, (size_t)c->sm_count * 8);
    k_merge_splits<U, XF><<<std::max(sg, 1), 256, 0, c->stream>>>(a, na, b, nb, tiles, split);
    ++c->launches;
    const int parts = sliced ? PIPE_SLICES : 1;
    for (int p = 0; p < parts; ++p) {
        const size_t t0 = tiles * p / parts, t1 = tiles * (p + 1) / parts;
        if (t1 > t0) {
            const int grid = (int)std::min<size_t>(t1 - t0, (size_t)c->sm_count * 8);
            k_merge_tiles<U, XF><<<grid, MERGE_THREADS, 0, c->stream>>>(a, na, b, nb, out, split, t0, t1);
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

template <typename U, int XF>
ts_status pipeline_body(ts_ctx* c, U* h, size_t n) {
    const int C = c->transfer_chunks;
    ts_status s;
    if ((s = grow(c, c->keys, n * sizeof(U), "keys")) != TS_OK) return s;
    if ((s = grow(c, c->alt, n * sizeof(U), "scratch keys")) != TS_OK) return s;
    if ((s = grow(c, c->pipe, ((n + MERGE_TILE - 1) / MERGE_TILE + 1) * sizeof(size_t), "merge splits")) != TS_OK)
        return s;
    if ((s = pipe_resources(c, (size_t)C + PIPE_SLICES + 2)) != TS_OK) return s;
    cudaPointerAttributes pa{};
    bool pageable = cudaPointerGetAttributes(&pa, h) != cudaSuccess || pa.type == cudaMemoryTypeUnregistered;
    cudaGetLastError();
    if (pageable && !stage_resources(c)) pageable = false;
    char* stage = (char*)c->stage;
    int slot = 0;
    // staged copy in of h[b, e): each slot waits for its previous DMA, is
    // filled by the copy threads, then goes to the device
    auto staged_in = [&](U* dst, const U* src, size_t count) -> ts_status {
        const size_t per = STAGE_SLOT_BYTES / sizeof(U);
        for (size_t q = 0; q < count; q += per) {
            const size_t m = std::min(per, count - q);
            TS_CUDA(c, cudaEventSynchronize(c->stage_events[slot]));
            char* buf = stage + (size_t)slot * STAGE_SLOT_BYTES;
            c->copy_pool->copy(buf, src + q, m * sizeof(U));
            TS_CUDA(c, cudaMemcpyAsync(dst + q, buf, m * sizeof(U), cudaMemcpyHostToDevice, c->copy_stream));
            TS_CUDA(c, cudaEventRecord(c->stage_events[slot], c->copy_stream));
            slot = (slot + 1) % STAGE_SLOTS;
        }
        return TS_OK;
    };
    U* X = (U*)c->keys.p;
    U* Y = (U*)c->alt.p;
    const size_t chunk = ((n + C - 1) / C + 255) / 256 * 256;  // chunk starts 256 keys apart: 16-byte aligned
    auto lo = [&](int i) { return std::min(n, (size_t)i * chunk); };
    cudaEvent_t* in_ev = c->pipe_events.data();         // [C] chunk i is on the device
    cudaEvent_t* out_ev = in_ev + C;                    // [PIPE_SLICES] output slice p is merged
    cudaEvent_t ready_ev = in_ev[C + PIPE_SLICES];      // the context's stream reached this call
    cudaEvent_t done_ev = in_ev[C + PIPE_SLICES + 1];   // the last copy out ended

    // the copies start behind whatever the context's stream already holds
    TS_CUDA(c, cudaEventRecord(ready_ev, c->stream));
    TS_CUDA(c, cudaStreamWaitEvent(c->copy_stream, ready_ev, 0));
    auto copy_in = [&](int i) -> ts_status {
        if (i >= C) return TS_OK;
        const size_t b = lo(i), e = lo(i + 1);
        if (e > b) {
            if (pageable) {
                ts_status st = staged_in(X + b, h + b, e - b);
                if (st != TS_OK) return st;
            } else {
                TS_CUDA(c, cudaMemcpyAsync(X + b, h + b, (e - b) * sizeof(U), cudaMemcpyHostToDevice, c->copy_stream));
            }
        }
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
    size_t slice_end[PIPE_SLICES] = {};
    U* final_buf = X;
    for (int i = 0; i < C; ++i) {
        TS_CUDA(c, cudaStreamWaitEvent(c->stream, in_ev[i], 0));
        const size_t b = lo(i), e = lo(i + 1);
        if ((s = sort_keys_device<U, XF>(c, X + b, e - b, Y + b)) != TS_OK) return s;
        runs.push_back({b, e, 0});
        while (runs.size() >= 2 && runs[runs.size() - 1].level == runs[runs.size() - 2].level) {
            const Run r2 = runs.back();
            runs.pop_back();
            const Run r1 = runs.back();
            runs.pop_back();
            const int L = r1.level;
            U* src = (L & 1) ? Y : X;
            U* dst = (L & 1) ? X : Y;
            const bool last = i == C - 1 && runs.empty();
            mark(c, "merge");
            if ((s = enqueue_merge<U, XF>(c, src + r1.b, r1.e - r1.b, src + r2.b, r2.e - r2.b, dst + r1.b, last, out_ev,
                                          slice_end)) != TS_OK)
                return s;
            runs.push_back({r1.b, r2.e, L + 1});
            if (last) final_buf = dst;
        }
        if ((s = copy_in(i + 2)) != TS_OK) return s;
    }
    mark(c, "end");
    // the sorted slice goes back one merged output slice at a time
    if (!pageable) {
        size_t from = 0;
        for (int p = 0; p < PIPE_SLICES; ++p) {
            TS_CUDA(c, cudaStreamWaitEvent(c->copy_stream, out_ev[p], 0));
            if (slice_end[p] > from)
                TS_CUDA(c, cudaMemcpyAsync(h + from, final_buf + from, (slice_end[p] - from) * sizeof(U),
                                           cudaMemcpyDeviceToHost, c->copy_stream));
            from = std::max(from, slice_end[p]);
        }
    } else {
        // pieces of at most one slot, none across a slice end; the DMA of
        // piece k + STAGE_SLOTS - 1 is queued before the threads empty piece k
        struct Piece {
            size_t b, e;
            int slice;
        };
        std::vector<Piece> pieces;
        const size_t per = STAGE_SLOT_BYTES / sizeof(U);
        size_t from = 0;
        for (int p = 0; p < PIPE_SLICES; ++p) {
            for (size_t q = from; q < slice_end[p]; q += per) pieces.push_back({q, std::min(slice_end[p], q + per), p});
            from = std::max(from, slice_end[p]);
        }
        int waited = -1;  // the last slice the copy stream waits for
        auto issue = [&](size_t k) -> ts_status {
            const Piece& pc = pieces[k];
            for (; waited < pc.slice; ++waited) TS_CUDA(c, cudaStreamWaitEvent(c->copy_stream, out_ev[waited + 1], 0));
            const int sl = (int)(k % STAGE_SLOTS);
            TS_CUDA(c, cudaMemcpyAsync(stage + (size_t)sl * STAGE_SLOT_BYTES, final_buf + pc.b, (pc.e - pc.b) * sizeof(U),
                                       cudaMemcpyDeviceToHost, c->copy_stream));
            TS_CUDA(c, cudaEventRecord(c->stage_events[sl], c->copy_stream));
            return TS_OK;
        };
        for (size_t k = 0; k + 1 < (size_t)STAGE_SLOTS && k < pieces.size(); ++k)
            if ((s = issue(k)) != TS_OK) return s;
        for (size_t k = 0; k < pieces.size(); ++k) {
            if (k + STAGE_SLOTS - 1 < pieces.size())
                if ((s = issue(k + STAGE_SLOTS - 1)) != TS_OK) return s;
            const int sl = (int)(k % STAGE_SLOTS);
            TS_CUDA(c, cudaEventSynchronize(c->stage_events[sl]));
            c->copy_pool->copy(h + pieces[k].b, stage + (size_t)sl * STAGE_SLOT_BYTES,
                               (pieces[k].e - pieces[k].b) * sizeof(U));
        }
    }
    TS_CUDA(c, cudaEventRecord(done_ev, c->copy_stream));
    TS_CUDA(c, cudaStreamWaitEvent(c->stream, done_ev, 0));
    return TS_OK;
}

// Sort the host slice h[0, n) with the copies overlapped (c->transfer_chunks
// a power of two, at least 2). Returns once the sorted keys are back in h.
template <typename U, int XF>
ts_status pipeline_sort(ts_ctx* c, U* h, size_t n) {
    ts_status s = pipeline_body<U, XF>(c, h, n);
    if (s != TS_OK) {
        // nothing may still be copying into or out of the caller's slice
        if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);
        cudaStreamSynchronize(c->stream);
        return s;
    }
    return finish(c);
}

}  // namespace ts
