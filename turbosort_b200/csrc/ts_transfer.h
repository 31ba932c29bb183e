// ts_transfer.h — the copies of a pipelined host-slice call: two copy
// streams beside the context's stream (copies in, and copies out that must
// run while copies in continue), events, and for pageable host memory the
// context's pinned staging slots with the copy pool's threads (ts_staging.h).
//
// A pageable host slice cannot be a DMA source or target; the CUDA driver would
// copy it through its own pinned buffer on the calling thread at about a
// quarter of the PCIe rate. Such a slice goes through STAGE_SLOTS pinned
// slots instead: the copy threads fill a slot while the DMA of the previous
// one runs, and on the way back empty a slot while the next ones' DMAs run.
// Each slot's reuse waits for its last DMA (an event), in either direction.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "ts_ctx.h"
#include "ts_staging.h"

namespace ts {

constexpr int PIPE_SLICES = 8;                     // output slices of the last merge
constexpr int STAGE_SLOTS = 4;                     // pinned staging slots for pageable slices
constexpr size_t STAGE_SLOT_BYTES = (size_t)32 << 20;

// the pinned slots, their events and the copy threads; false if pinned
// memory cannot be had (the slice then takes the CUDA driver's own staging)
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
    if (!c->out_stream) TS_CUDA(c, cudaStreamCreateWithFlags(&c->out_stream, cudaStreamNonBlocking));
    while (c->pipe_events.size() < events) {
        cudaEvent_t ev;
        TS_CUDA(c, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        c->pipe_events.push_back(ev);
    }
    return TS_OK;
}

// the events a pipelined call records: [C] chunks in, [PIPE_SLICES] output
// slices merged, then "stream reached the call" and "copies out done"
inline cudaEvent_t* slice_events(ts_ctx* c) { return c->pipe_events.data() + c->transfer_chunks; }
inline cudaEvent_t done_event(ts_ctx* c) { return c->pipe_events[c->transfer_chunks + PIPE_SLICES + 1]; }

// whatever failed, nothing may still copy into or out of the caller's slices
inline ts_status pipeline_end(ts_ctx* c, ts_status s) {
    if (s != TS_OK) {
        if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);
        if (c->out_stream) cudaStreamSynchronize(c->out_stream);
        cudaStreamSynchronize(c->stream);
        return s;
    }
    return finish(c);
}

// The copies of one pipelined call, on the copy stream: straight DMAs for a
// pinned (or registered) host slice, the staging slots for a pageable one.
struct Transfer {
    ts_ctx* c;
    cudaStream_t st;
    bool pageable = false;
    int slot = 0;

    // st: the stream the copies go on (the context's copy stream by default)
    Transfer(ts_ctx* ctx, const void* host, cudaStream_t stream = nullptr)
        : c(ctx), st(stream ? stream : ctx->copy_stream) {
        cudaPointerAttributes pa{};
        pageable = cudaPointerGetAttributes(&pa, host) != cudaSuccess || pa.type == cudaMemoryTypeUnregistered;
        cudaGetLastError();
        if (pageable && !stage_resources(c)) pageable = false;
    }

    // host[0, bytes) to dev: each slot waits for its previous DMA, is filled
    // by the copy threads, then goes to the device
    ts_status in(void* dev, const void* host, size_t bytes) {
        if (bytes == 0) return TS_OK;
        if (!pageable) {
            TS_CUDA(c, cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, st));
            return TS_OK;
        }
        for (size_t q = 0; q < bytes; q += STAGE_SLOT_BYTES) {
            const size_t m = std::min(STAGE_SLOT_BYTES, bytes - q);
            TS_CUDA(c, cudaEventSynchronize(c->stage_events[slot]));
            char* buf = (char*)c->stage + (size_t)slot * STAGE_SLOT_BYTES;
            c->copy_pool->copy(buf, (const char*)host + q, m);
            TS_CUDA(c, cudaMemcpyAsync((char*)dev + q, buf, m, cudaMemcpyHostToDevice, st));
            TS_CUDA(c, cudaEventRecord(c->stage_events[slot], st));
            slot = (slot + 1) % STAGE_SLOTS;
        }
        return TS_OK;
    }

    // dev to host, slice by slice: slice p (bytes up to end[p]) once
    // slice_ev[p] has happened on the context's stream. Pageable: pieces of
    // at most one slot, none across a slice end; the DMA of piece
    // k + STAGE_SLOTS - 1 is queued before the threads empty piece k.
    ts_status out(void* host, const void* dev, const size_t* end, cudaEvent_t* slice_ev, int slices) {
        if (!pageable) {
            size_t from = 0;
            for (int p = 0; p < slices; ++p) {
                TS_CUDA(c, cudaStreamWaitEvent(st, slice_ev[p], 0));
                if (end[p] > from)
                    TS_CUDA(c, cudaMemcpyAsync((char*)host + from, (const char*)dev + from, end[p] - from,
                                               cudaMemcpyDeviceToHost, st));
                from = std::max(from, end[p]);
            }
            return TS_OK;
        }
        struct Piece {
            size_t b, e;
            int slice;
        };
        std::vector<Piece> pieces;
        size_t from = 0;
        for (int p = 0; p < slices; ++p) {
            for (size_t q = from; q < end[p]; q += STAGE_SLOT_BYTES)
                pieces.push_back({q, std::min(end[p], q + STAGE_SLOT_BYTES), p});
            from = std::max(from, end[p]);
        }
        int waited = -1;  // the last slice the copy stream waits for
        auto issue = [&](size_t k) -> ts_status {
            const Piece& pc = pieces[k];
            for (; waited < pc.slice; ++waited) TS_CUDA(c, cudaStreamWaitEvent(st, slice_ev[waited + 1], 0));
            const int sl = (int)(k % STAGE_SLOTS);
            // the slot's last DMA (in either direction, on any stream) is done
            TS_CUDA(c, cudaStreamWaitEvent(st, c->stage_events[sl], 0));
            TS_CUDA(c, cudaMemcpyAsync((char*)c->stage + (size_t)sl * STAGE_SLOT_BYTES, (const char*)dev + pc.b,
                                       pc.e - pc.b, cudaMemcpyDeviceToHost, st));
            TS_CUDA(c, cudaEventRecord(c->stage_events[sl], st));
            return TS_OK;
        };
        ts_status s;
        for (size_t k = 0; k + 1 < (size_t)STAGE_SLOTS && k < pieces.size(); ++k)
            if ((s = issue(k)) != TS_OK) return s;
        for (size_t k = 0; k < pieces.size(); ++k) {
            if (k + STAGE_SLOTS - 1 < pieces.size())
                if ((s = issue(k + STAGE_SLOTS - 1)) != TS_OK) return s;
            const int sl = (int)(k % STAGE_SLOTS);
            TS_CUDA(c, cudaEventSynchronize(c->stage_events[sl]));
            c->copy_pool->copy((char*)host + pieces[k].b, (const char*)c->stage + (size_t)sl * STAGE_SLOT_BYTES,
                               pieces[k].e - pieces[k].b);
        }
        return TS_OK;
    }
};

}  // namespace ts
