// ts_ctx.h — the context behind the C ABI: one CUDA stream, grow-only device
// scratch (the GPU counterpart of the crate's scratch buffers and of
// SortByKeyBuffer, src/by_key.rs:51-90), the error word the kernels report
// through, and optional per-kernel CUDA-event timing.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <string>
#include <utility>
#include <vector>

#include "../../include/turbosort.h"

namespace ts {

struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
};
class CopyPool;

}  // namespace ts

struct ts_ctx {
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    bool own_stream = false;

    // grow-only device buffers
    ts::DevBuf keys, alt;          // staged keys and their ping-pong partner
    ts::DevBuf vals0, vals1;       // positions ping-pong (sort_by_key)
    ts::DevBuf order;              // the order of the last sort_by_key
    ts::DevBuf meta;               // scan state, plan, histograms, scans, counters, carries
    ts::DevBuf lookback;           // two look-back regions
    ts::DevBuf runs;               // a diverted sort's list of long runs
    ts::DevBuf gather;             // apply_order staging
    ts::DevBuf seg;                // segmented sort: plan, work counter, bin lists, offsets
    ts::DevBuf learn;              // learned partition: sample, model, training state, bucket counts
    ts::DevBuf check;              // learned partition's verify pass: a copy of the keys, sorted by the plain LSD
    ts::DevBuf pipe;               // host-slice pipeline: merge split points
    ts::DevBuf pipe_pos[2];        // host-slice pipeline of sort_by_key: position runs
    uint32_t* d_error = nullptr;   // kernel-reported errors, read and cleared by the host

    // plain LSD: the tile variant (k_onesweep keys a thread, halved per step)
    // per key width (1, 2, 4, 8 bytes) and length bin (< 2^22, < 2^25, more),
    // set by ts_lsd_autotune; the defaults were measured on a B200
    int lsd_variant[4][3] = {{0, 0, 0}, {1, 0, 0}, {1, 0, 0}, {0, 0, 0}};
    // the plain LSD's digit width per key width and length bin (4..11 bits)
    int lsd_bits[4][3] = {{8, 8, 8}, {8, 8, 8}, {8, 8, 8}, {8, 8, 8}};
    // segmented sort: the method of each on-chip length bin per key width
    // (1, 2, 4, 8 bytes), set by the autotuner; and the last captured graph
    int seg_methods[4][4] = {{4, 5, 2, 2}, {4, 5, 2, 2}, {4, 5, 6, 6}, {4, 3, 6, 6}};
    bool use_graphs = true;
    bool capturing = false;
    cudaGraphExec_t seg_graph = nullptr;
    size_t seg_graph_key[10] = {};
    // plain device sort: the launch sequence of a repeated call, captured on
    // its second identical call and replayed afterwards
    cudaGraphExec_t sort_graph = nullptr;
    size_t sort_graph_key[9] = {};
    size_t sort_last_key[9] = {};
    unsigned long long sort_graph_launches = 0;

    // host-slice sorts of at least transfer_min_bytes cross as transfer_chunks
    // pieces on copy_stream, sorted and merged while the copies run
    int transfer_chunks = 8;
    size_t transfer_min_bytes = (size_t)64 << 20;
    cudaStream_t copy_stream = nullptr;
    cudaStream_t out_stream = nullptr;     // copies back that overlap copies in
    std::vector<cudaEvent_t> pipe_events;
    // pageable host slices go through pinned staging slots, filled and
    // emptied by the copy pool's threads
    void* stage = nullptr;                 // pinned host memory: STAGE_SLOTS slots
    std::vector<cudaEvent_t> stage_events; // the last DMA of each slot
    ts::CopyPool* copy_pool = nullptr;

    // diverting of 8-byte keys (ts_ctx_set_divert), on by default as in the crate
    bool divert = true;
    // 2- and 4-byte keys whose tiles fit one wave sort in one cooperative
    // launch (ts_ctx_set_single_launch)
    bool coop = true;
    // test hook (ts_ctx_test_stall_lookback): the next LSD sort's first pass
    // withholds tile 0's look-back entry and gives up after this many rounds
    uint32_t test_spin_limit = 0;
    // the tier of the last plain sort (ts_sort_info: 1 small, 2 counting, 3 LSD,
    // 4 LSD in one launch)
    int last_tier = 0;
    int last_bits = 8;  // the last LSD sort's digit width

    std::string last_error;
    unsigned long long launches = 0;   // kernels this context has launched

    // timing: named marks on the stream, folded into per-name totals on read
    bool timing = false;
    std::vector<std::pair<std::string, cudaEvent_t>> marks;
    std::vector<cudaEvent_t> spare_events;
    std::map<std::string, std::pair<double, long>> totals;
};

namespace ts {

// Record a named mark: the time until the next mark is charged to `name`.
void mark(ts_ctx* c, const char* name);
// Fold the recorded marks into totals (synchronises on the last mark).
void fold_marks(ts_ctx* c);

ts_status fail(ts_ctx* c, ts_status s, const std::string& msg);
// Wait for the context's stream and report what the kernels flagged.
ts_status finish(ts_ctx* c);
ts_status cuda_fail(ts_ctx* c, cudaError_t e, const char* where);
ts_status grow(ts_ctx* c, DevBuf& b, size_t bytes, const char* what);

// Device sorts, enqueued on c->stream. The caller checks the error word.
template <typename U, int XF>
ts_status sort_keys_device(ts_ctx* c, U* d_data, size_t n, U* d_alt);
template <typename U, int XF>
ts_status order_device(ts_ctx* c, const U* d_keys, size_t n, uint32_t* d_order);
// The host slice h[0, n) sorted with its copies overlapped; returns when done.
template <typename U, int XF>
ts_status pipeline_sort(ts_ctx* c, U* h, size_t n);
// The stable order of the host keys h_keys[0, n) with the copies overlapped.
template <typename U, int XF>
ts_status pipeline_order(ts_ctx* c, const U* h_keys, size_t n, uint32_t* h_order);

}  // namespace ts

#define TS_CUDA(c, call)                                        \
    do {                                                        \
        cudaError_t e_ = (call);                                \
        if (e_ != cudaSuccess) return ts::cuda_fail((c), e_, #call); \
    } while (0)
