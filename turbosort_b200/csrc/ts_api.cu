// ts_api.cu — the C ABI (include/turbosort.h): contexts, the per-type entry
// points that replace the crate's public functions, apply_order, timing.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <unordered_map>

#include "ts_ctx.h"
#include "ts_engine.cuh"
#include "ts_gather.cuh"
#include "ts_transfer.h"

namespace ts {

ts_status fail(ts_ctx* c, ts_status s, const std::string& msg) {
    if (c) c->last_error = msg;
    return s;
}

ts_status cuda_fail(ts_ctx* c, cudaError_t e, const char* where) {
    std::string msg = std::string(where) + ": " + cudaGetErrorString(e);
    return fail(c, e == cudaErrorMemoryAllocation ? TS_ERR_OOM : TS_ERR_CUDA, msg);
}

ts_status grow(ts_ctx* c, DevBuf& b, size_t bytes, const char* what) {
    if (bytes <= b.cap) return TS_OK;
    if (b.p) {
        // the stream may still use the old buffer
        cudaError_t e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) return cuda_fail(c, e, "cudaStreamSynchronize");
        cudaFree(b.p);
        b.p = nullptr;
        b.cap = 0;
    }
    size_t want = (bytes + 4095) / 4096 * 4096;
    cudaError_t e = cudaMalloc(&b.p, want);
    if (e != cudaSuccess) {
        b.p = nullptr;
        cudaGetLastError();
        return fail(c, TS_ERR_OOM, std::string("cannot reserve ") + std::to_string(want) + " bytes for " + what);
    }
    b.cap = want;
    return TS_OK;
}

int occupancy_of(const void* kernel, int threads, size_t smem) {
    static std::mutex mu;
    static std::unordered_map<const void*, int> cache;
    std::lock_guard<std::mutex> g(mu);
    auto it = cache.find(kernel);
    if (it != cache.end()) return it->second;
    // the default limit (48 KB) covers static and dynamic shared memory together
    cudaFuncAttributes fa{};
    if (cudaFuncGetAttributes(&fa, kernel) != cudaSuccess) cudaGetLastError();
    if (smem + fa.sharedSizeBytes > 48 * 1024)
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int blocks = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kernel, threads, smem);
    if (blocks < 1) blocks = 1;
    cache[kernel] = blocks;
    return blocks;
}

void mark(ts_ctx* c, const char* name) {
    if (!c->timing || c->capturing) return;
    cudaEvent_t ev;
    if (!c->spare_events.empty()) {
        ev = c->spare_events.back();
        c->spare_events.pop_back();
    } else if (cudaEventCreate(&ev) != cudaSuccess) {
        return;
    }
    cudaEventRecord(ev, c->stream);
    c->marks.emplace_back(name, ev);
}

void fold_marks(ts_ctx* c) {
    if (c->marks.empty()) return;
    cudaEventSynchronize(c->marks.back().second);
    for (size_t i = 0; i + 1 < c->marks.size(); ++i) {
        const std::string& name = c->marks[i].first;
        if (name == "end") continue;
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, c->marks[i].second, c->marks[i + 1].second) == cudaSuccess) {
            auto& t = c->totals[name];
            t.first += ms;
            t.second += 1;
        }
    }
    for (auto& m : c->marks) c->spare_events.push_back(m.second);
    c->marks.clear();
}

// Wait for the stream, then report what the kernels flagged.
ts_status finish(ts_ctx* c) {
    uint32_t host_err = 0;
    cudaError_t e = cudaMemcpyAsync(&host_err, c->d_error, 4, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(c->d_error, 0, 4, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "synchronize");
    if (c->timing) {
        mark(c, "end");
        fold_marks(c);
    }
    if (host_err & ERR_TIMEOUT)
        return fail(c, TS_ERR_TIMEOUT, "a bounded wait in the onesweep look-back ran out; output not valid");
    if (host_err & ERR_BOUNDS) return fail(c, TS_ERR_INTERNAL, "a device-side bounds check fired");
    return TS_OK;
}

// ---- host-slice entry points -------------------------------------------------

template <typename T, typename U, int XF>
static ts_status host_sort(ts_ctx* c, T* data, size_t n) {
    if (!c) return TS_ERR_INVALID;
    if (n <= 1) return TS_OK;
    if (!data) return fail(c, TS_ERR_INVALID, "null data");
    if constexpr (sizeof(U) > 1) {
        if (c->transfer_chunks > 1 && n * sizeof(U) >= c->transfer_min_bytes && n >= (size_t)c->transfer_chunks * 256)
            return pipeline_sort<U, XF>(c, (U*)data, n);
    }
    ts_status s;
    if ((s = grow(c, c->keys, n * sizeof(U), "keys")) != TS_OK) return s;
    U* d = (U*)c->keys.p;
    mark(c, "h2d");
    TS_CUDA(c, cudaMemcpyAsync(d, data, n * sizeof(U), cudaMemcpyHostToDevice, c->stream));
    if ((s = sort_keys_device<U, XF>(c, d, n, nullptr)) != TS_OK) return s;
    mark(c, "d2h");
    TS_CUDA(c, cudaMemcpyAsync(data, d, n * sizeof(U), cudaMemcpyDeviceToHost, c->stream));
    return finish(c);
}

static ts_status buffer_check(ts_ctx* c, size_t n, size_t buf_len) {
    if (buf_len < n) {
        char msg[96];
        snprintf(msg, sizeof msg, "buffer too small: need %zu, got %zu", n, buf_len);
        return fail(c, TS_ERR_BUFFER_TOO_SMALL, msg);
    }
    return TS_OK;
}

template <typename T, typename U, int XF>
static ts_status host_order(ts_ctx* c, const T* keys, size_t n, uint32_t* order) {
    if (!c) return TS_ERR_INVALID;
    if (n > 0xffffffffull) return fail(c, TS_ERR_TOO_LARGE, "sort_by_key: more than u32::MAX elements");
    if (n == 0) return TS_OK;
    if (!keys || !order) return fail(c, TS_ERR_INVALID, "null keys or order");
    if (n == 1) {
        order[0] = 0;
        return TS_OK;
    }
    if constexpr (sizeof(U) > 1) {
        if (c->transfer_chunks > 1 && n * (sizeof(U) + 4) >= c->transfer_min_bytes &&
            n >= (size_t)c->transfer_chunks * 256)
            return pipeline_order<U, XF>(c, (const U*)keys, n, order);
    }
    ts_status s;
    if ((s = grow(c, c->keys, n * sizeof(U), "keys")) != TS_OK) return s;
    if ((s = grow(c, c->order, n * 4, "order")) != TS_OK) return s;
    mark(c, "h2d");
    TS_CUDA(c, cudaMemcpyAsync(c->keys.p, keys, n * sizeof(U), cudaMemcpyHostToDevice, c->stream));
    if ((s = order_device<U, XF>(c, (const U*)c->keys.p, n, (uint32_t*)c->order.p)) != TS_OK) return s;
    mark(c, "d2h");
    TS_CUDA(c, cudaMemcpyAsync(order, c->order.p, n * 4, cudaMemcpyDeviceToHost, c->stream));
    return finish(c);
}

template <typename U, int XF>
static ts_status dev_sort(ts_ctx* c, U* d, size_t n, U* alt) {
    if (!c) return TS_ERR_INVALID;
    if (n <= 1) return TS_OK;
    if (!d) return fail(c, TS_ERR_INVALID, "null data");
    return sort_keys_device<U, XF>(c, d, n, alt);
}

template <typename U, int XF>
static ts_status dev_order(ts_ctx* c, const U* d, size_t n, uint32_t* order) {
    if (!c) return TS_ERR_INVALID;
    if (n > 0xffffffffull) return fail(c, TS_ERR_TOO_LARGE, "sort_by_key: more than u32::MAX elements");
    if (n == 0) return TS_OK;
    if (!d || !order) return fail(c, TS_ERR_INVALID, "null keys or order");
    if (n == 1) {
        TS_CUDA(c, cudaMemsetAsync(order, 0, 4, c->stream));
        return TS_OK;
    }
    return order_device<U, XF>(c, d, n, order);
}

// out[i] = in[order[i]] for i < n, elements of `elem` bytes; order[i] < n_src
static ts_status gather_dev(ts_ctx* c, const void* in, void* out, const uint32_t* order, size_t n, size_t elem,
                            size_t n_src) {
    const int grid = c->sm_count * 8;
    if (elem % 16 == 0 && ((uintptr_t)in & 15) == 0 && ((uintptr_t)out & 15) == 0) {
        k_gather<uint4><<<grid, 256, 0, c->stream>>>((const uint4*)in, (uint4*)out, order, n, n_src,
                                                     (uint32_t)(elem / 16), c->d_error);
    } else if (elem % 8 == 0 && ((uintptr_t)in & 7) == 0 && ((uintptr_t)out & 7) == 0) {
        k_gather<uint2><<<grid, 256, 0, c->stream>>>((const uint2*)in, (uint2*)out, order, n, n_src,
                                                     (uint32_t)(elem / 8), c->d_error);
    } else if (elem % 4 == 0 && ((uintptr_t)in & 3) == 0 && ((uintptr_t)out & 3) == 0) {
        k_gather<uint32_t><<<grid, 256, 0, c->stream>>>((const uint32_t*)in, (uint32_t*)out, order, n, n_src,
                                                        (uint32_t)(elem / 4), c->d_error);
    } else {
        k_gather<uint8_t><<<grid, 256, 0, c->stream>>>((const uint8_t*)in, (uint8_t*)out, order, n, n_src,
                                                       (uint32_t)elem, c->d_error);
    }
    ++c->launches;
    TS_CUDA(c, cudaGetLastError());
    return TS_OK;
}

// Host apply_order with its copies overlapped: the order and the elements
// cross on the copy stream (through the staging slots when pageable), the
// gather runs in PIPE_SLICES output slices, and each slice goes back while
// the next is gathered.
static ts_status pipeline_apply_order(ts_ctx* c, void* data, size_t n, size_t elem, const uint32_t* order) {
    const size_t bytes = n * elem;
    const size_t half = (bytes + 255) / 256 * 256;
    ts_status s;
    if ((s = grow(c, c->gather, 2 * half, "apply_order staging")) != TS_OK) return s;
    if ((s = grow(c, c->order, n * 4, "order")) != TS_OK) return s;
    if ((s = pipe_resources(c, (size_t)c->transfer_chunks + PIPE_SLICES + 2)) != TS_OK) return s;
    char* a = (char*)c->gather.p;
    char* b = a + half;
    uint32_t* d_order = (uint32_t*)c->order.p;
    cudaEvent_t* ev = c->pipe_events.data();
    Transfer to(c, order), td(c, data);
    mark(c, "h2d");
    TS_CUDA(c, cudaEventRecord(ev[0], c->stream));
    TS_CUDA(c, cudaStreamWaitEvent(c->copy_stream, ev[0], 0));
    if ((s = to.in(d_order, order, n * 4)) != TS_OK) return s;
    td.slot = to.slot;
    if ((s = td.in(a, data, bytes)) != TS_OK) return s;
    TS_CUDA(c, cudaEventRecord(ev[1], c->copy_stream));
    TS_CUDA(c, cudaStreamWaitEvent(c->stream, ev[1], 0));
    mark(c, "gather");
    size_t end[PIPE_SLICES];
    cudaEvent_t* slice_ev = slice_events(c);
    for (int p = 0; p < PIPE_SLICES; ++p) {
        // slice starts 256 elements apart keep every slice's output aligned
        const size_t lo = p == 0 ? 0 : std::min(n, n * p / PIPE_SLICES / 256 * 256);
        const size_t hi = p + 1 == PIPE_SLICES ? n : std::min(n, n * (p + 1) / PIPE_SLICES / 256 * 256);
        if (hi > lo && (s = gather_dev(c, a, b + lo * elem, d_order + lo, hi - lo, elem, n)) != TS_OK) return s;
        end[p] = hi * elem;
        TS_CUDA(c, cudaEventRecord(slice_ev[p], c->stream));
    }
    mark(c, "end");
    if ((s = td.out(data, b, end, slice_ev, PIPE_SLICES)) != TS_OK) return s;
    TS_CUDA(c, cudaEventRecord(done_event(c), c->copy_stream));
    TS_CUDA(c, cudaStreamWaitEvent(c->stream, done_event(c), 0));
    return TS_OK;
}

}  // namespace ts

using namespace ts;

extern "C" {

ts_status ts_ctx_create(int device, ts_ctx** out) {
    if (!out) return TS_ERR_INVALID;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return TS_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= count) return TS_ERR_INVALID;
    if (cudaSetDevice(device) != cudaSuccess) return TS_ERR_CUDA;
    ts_ctx* c = new ts_ctx();
    c->device = device;
    cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device);
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&c->d_error, 256) != cudaSuccess || cudaMemset(c->d_error, 0, 256) != cudaSuccess) {
        cudaGetLastError();
        delete c;
        return TS_ERR_CUDA;
    }
    c->own_stream = true;
    *out = c;
    return TS_OK;
}

void ts_ctx_destroy(ts_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);
    if (c->out_stream) cudaStreamSynchronize(c->out_stream);
    for (DevBuf* b : {&c->keys, &c->alt, &c->vals0, &c->vals1, &c->order, &c->meta, &c->lookback, &c->runs, &c->gather,
                      &c->seg, &c->check,
                      &c->learn, &c->pipe, &c->pipe_pos[0], &c->pipe_pos[1]})
        if (b->p) cudaFree(b->p);
    for (auto ev : c->pipe_events) cudaEventDestroy(ev);
    for (auto ev : c->stage_events) cudaEventDestroy(ev);
    if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
    if (c->out_stream) cudaStreamDestroy(c->out_stream);
    if (c->stage) cudaFreeHost(c->stage);
    delete c->copy_pool;
    if (c->seg_graph) cudaGraphExecDestroy(c->seg_graph);
    if (c->sort_graph) cudaGraphExecDestroy(c->sort_graph);
    if (c->d_error) cudaFree(c->d_error);
    for (auto& m : c->marks) cudaEventDestroy(m.second);
    for (auto ev : c->spare_events) cudaEventDestroy(ev);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

ts_status ts_ctx_set_stream(ts_ctx* c, void* stream) {
    if (!c) return TS_ERR_INVALID;
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    c->stream = (cudaStream_t)stream;
    c->own_stream = false;
    return TS_OK;
}

void* ts_ctx_stream(ts_ctx* c) { return c ? (void*)c->stream : nullptr; }

ts_status ts_ctx_transfer_pipeline(ts_ctx* c, int chunks, size_t min_bytes) {
    if (!c) return TS_ERR_INVALID;
    if (chunks < 1 || chunks > 64 || (chunks & (chunks - 1)) != 0)
        return fail(c, TS_ERR_INVALID, "transfer chunks must be a power of two from 1 to 64");
    c->transfer_chunks = chunks;
    c->transfer_min_bytes = min_bytes;
    return TS_OK;
}

ts_status ts_ctx_synchronize(ts_ctx* c) {
    if (!c) return TS_ERR_INVALID;
    return finish(c);
}

ts_status ts_ctx_reserve(ts_ctx* c, size_t n, size_t key_bytes, int with_order) {
    if (!c) return TS_ERR_INVALID;
    ts_status s;
    if ((s = grow(c, c->keys, n * key_bytes, "keys")) != TS_OK) return s;
    if ((s = grow(c, c->alt, (with_order ? 2 : 1) * n * key_bytes + 16, "scratch keys")) != TS_OK) return s;
    if (with_order) {
        if ((s = grow(c, c->vals0, n * 4, "positions")) != TS_OK) return s;
        if ((s = grow(c, c->vals1, n * 4, "positions")) != TS_OK) return s;
        if ((s = grow(c, c->order, n * 4, "order")) != TS_OK) return s;
    }
    return TS_OK;
}

size_t ts_ctx_capacity(const ts_ctx* c, size_t key_bytes, int with_order) {
    if (!c || key_bytes == 0) return 0;
    size_t cap = c->keys.cap / key_bytes;
    if (with_order) {
        cap = std::min(cap, c->alt.cap / (2 * key_bytes));
        cap = std::min(cap, std::min(c->vals0.cap, std::min(c->vals1.cap, c->order.cap)) / 4);
    } else {
        cap = std::min(cap, c->alt.cap / key_bytes);
    }
    return cap;
}

const char* ts_ctx_last_error(const ts_ctx* c) { return c ? c->last_error.c_str() : "null context"; }

const char* ts_status_str(ts_status s) {
    switch (s) {
        case TS_OK: return "ok";
        case TS_ERR_BUFFER_TOO_SMALL: return "buffer too small";
        case TS_ERR_LENGTH_MISMATCH: return "length mismatch";
        case TS_ERR_CUDA: return "CUDA error";
        case TS_ERR_TIMEOUT: return "device wait timed out";
        case TS_ERR_OOM: return "out of device memory";
        case TS_ERR_INVALID: return "invalid argument";
        case TS_ERR_NO_DEVICE: return "no CUDA device";
        case TS_ERR_TOO_LARGE: return "too many elements";
        case TS_ERR_INTERNAL: return "internal bounds check";
    }
    return "unknown status";
}

ts_status ts_ctx_enable_timing(ts_ctx* c, int on) {
    if (!c) return TS_ERR_INVALID;
    c->timing = on != 0;
    return TS_OK;
}

int ts_ctx_timings(ts_ctx* c, char (*names)[32], double* ms, long* counts, int max) {
    if (!c) return 0;
    if (!c->marks.empty()) {
        cudaStreamSynchronize(c->stream);
        mark(c, "end");
        fold_marks(c);
    }
    int i = 0;
    for (auto& kv : c->totals) {
        if (i < max) {
            if (names) {
                strncpy(names[i], kv.first.c_str(), 31);
                names[i][31] = 0;
            }
            if (ms) ms[i] = kv.second.first;
            if (counts) counts[i] = kv.second.second;
        }
        ++i;
    }
    return i;
}

void ts_ctx_reset_timings(ts_ctx* c) {
    if (!c) return;
    fold_marks(c);
    c->totals.clear();
}

unsigned long long ts_ctx_launches(const ts_ctx* c) { return c ? c->launches : 0ull; }

ts_status ts_ctx_last_sort_info(ts_ctx* c, ts_sort_info* info) {
    if (!c || !info) return TS_ERR_INVALID;
    std::memset(info, 0, sizeof *info);
    info->tier = c->last_tier;
    if ((c->last_tier != 3 && c->last_tier != 4) || !c->meta.p) return TS_OK;
    Plan p{};
    const MetaLayout m = MetaLayout::make(1, 1, 0);  // the plan's place does not depend on the sort
    TS_CUDA(c, cudaMemcpyAsync(&p, (const char*)c->meta.p + m.plan_off, sizeof p, cudaMemcpyDeviceToHost, c->stream));
    TS_CUDA(c, cudaStreamSynchronize(c->stream));
    info->mode = p.mode;
    info->passes = p.n_live;
    info->divert_shift = p.divert_shift;
    for (int i = 0; i < p.n_live && i < 16; ++i) info->pass_digit[i] = p.pass[i];
    info->digit_bits = c->last_bits;
    return TS_OK;
}

ts_status ts_ctx_set_divert(ts_ctx* c, int on) {
    if (!c) return TS_ERR_INVALID;
    c->divert = on != 0;
    return TS_OK;
}

ts_status ts_ctx_set_single_launch(ts_ctx* c, int on) {
    if (!c) return TS_ERR_INVALID;
    c->coop = on != 0;
    return TS_OK;
}

ts_status ts_ctx_test_stall_lookback(ts_ctx* c, uint32_t spin_limit) {
    if (!c) return TS_ERR_INVALID;
    c->test_spin_limit = spin_limit;
    return TS_OK;
}

int ts_divert_skippable_digits(int n_live, uint64_t len, const uint64_t* max_bucket) {
    if (n_live <= 0 || len == 0 || !max_bucket) return 0;
    return skippable_digits(n_live, (unsigned long long)len, (const unsigned long long*)max_bucket);
}

#define TS_DEFINE_SORTS(SUF, T, U, XF)                                                              \
    ts_status ts_sort_##SUF(ts_ctx* c, T* data, size_t n) { return host_sort<T, U, XF>(c, data, n); } \
    ts_status ts_sort_with_buffer_##SUF(ts_ctx* c, T* data, size_t n, T* buf, size_t buf_len) {      \
        if (!c) return TS_ERR_INVALID;                                                              \
        ts_status s = buffer_check(c, n, buf_len);                                                  \
        if (s != TS_OK) return s;                                                                   \
        (void)buf;                                                                                  \
        return host_sort<T, U, XF>(c, data, n);                                                     \
    }                                                                                               \
    ts_status ts_sort_parallel_##SUF(ts_ctx* c, T* data, size_t n) { return host_sort<T, U, XF>(c, data, n); } \
    ts_status ts_sort_keys_order_##SUF(ts_ctx* c, const T* keys, size_t n, uint32_t* order) {        \
        return host_order<T, U, XF>(c, keys, n, order);                                             \
    }                                                                                               \
    ts_status ts_sort_dev_##SUF(ts_ctx* c, T* d_data, size_t n) {                                  \
        return dev_sort<U, XF>(c, (U*)d_data, n, nullptr);                                          \
    }                                                                                               \
    ts_status ts_sort_dev_with_buffer_##SUF(ts_ctx* c, T* d_data, size_t n, T* d_buf, size_t buf_len) { \
        if (!c) return TS_ERR_INVALID;                                                              \
        ts_status s = buffer_check(c, n, buf_len);                                                  \
        if (s != TS_OK) return s;                                                                   \
        return dev_sort<U, XF>(c, (U*)d_data, n, n > 1 ? (U*)d_buf : nullptr);                      \
    }                                                                                               \
    ts_status ts_sort_keys_order_dev_##SUF(ts_ctx* c, const T* d_keys, size_t n, uint32_t* d_order) { \
        return dev_order<U, XF>(c, (const U*)d_keys, n, d_order);                                   \
    }

TS_DEFINE_SORTS(u8, uint8_t, uint8_t, 0)
TS_DEFINE_SORTS(u16, uint16_t, uint16_t, 0)
TS_DEFINE_SORTS(u32, uint32_t, uint32_t, 0)
TS_DEFINE_SORTS(u64, uint64_t, uint64_t, 0)
TS_DEFINE_SORTS(i8, int8_t, uint8_t, 1)
TS_DEFINE_SORTS(i16, int16_t, uint16_t, 1)
TS_DEFINE_SORTS(i32, int32_t, uint32_t, 1)
TS_DEFINE_SORTS(i64, int64_t, uint64_t, 1)
TS_DEFINE_SORTS(f32, float, uint32_t, 2)
TS_DEFINE_SORTS(f64, double, uint64_t, 2)

ts_status ts_apply_order(ts_ctx* c, void* data, size_t n, size_t elem, const uint32_t* order, size_t order_len) {
    if (!c) return TS_ERR_INVALID;
    if (n != order_len)
        return fail(c, TS_ERR_LENGTH_MISMATCH, "apply_order: the slice's length differs from the last sorted slice's");
    if (n == 0 || elem == 0) return TS_OK;
    if (!data || !order) return fail(c, TS_ERR_INVALID, "null data or order");
    const size_t bytes = n * elem;
    if (c->transfer_chunks > 1 && bytes + n * 4 >= c->transfer_min_bytes && n >= (size_t)PIPE_SLICES * 256)
        return pipeline_end(c, pipeline_apply_order(c, data, n, elem, order));
    const size_t half = (bytes + 255) / 256 * 256;
    ts_status s;
    if ((s = grow(c, c->gather, 2 * half, "apply_order staging")) != TS_OK) return s;
    if ((s = grow(c, c->order, n * 4, "order")) != TS_OK) return s;
    char* a = (char*)c->gather.p;
    char* b = a + half;
    mark(c, "h2d");
    TS_CUDA(c, cudaMemcpyAsync(a, data, bytes, cudaMemcpyHostToDevice, c->stream));
    TS_CUDA(c, cudaMemcpyAsync(c->order.p, order, n * 4, cudaMemcpyHostToDevice, c->stream));
    mark(c, "gather");
    if ((s = gather_dev(c, a, b, (const uint32_t*)c->order.p, n, elem, n)) != TS_OK) return s;
    mark(c, "d2h");
    TS_CUDA(c, cudaMemcpyAsync(data, b, bytes, cudaMemcpyDeviceToHost, c->stream));
    return finish(c);
}

ts_status ts_apply_order_dev(ts_ctx* c, void* d_data, size_t n, size_t elem, const uint32_t* d_order,
                             size_t order_len) {
    if (!c) return TS_ERR_INVALID;
    if (n != order_len)
        return fail(c, TS_ERR_LENGTH_MISMATCH, "apply_order: the slice's length differs from the last sorted slice's");
    if (n == 0 || elem == 0) return TS_OK;
    if (!d_data || !d_order) return fail(c, TS_ERR_INVALID, "null data or order");
    const size_t bytes = n * elem;
    ts_status s;
    if ((s = grow(c, c->gather, bytes, "apply_order staging")) != TS_OK) return s;
    mark(c, "gather");
    if ((s = gather_dev(c, d_data, c->gather.p, d_order, n, elem, n)) != TS_OK) return s;
    mark(c, "copy");
    TS_CUDA(c, cudaMemcpyAsync(d_data, c->gather.p, bytes, cudaMemcpyDeviceToDevice, c->stream));
    return TS_OK;
}

}  // extern "C"
