// ts_segments.cu — the segmented batch sort: device driver, CUDA-graph
// replay, the autotuner of the on-chip methods, and its C ABI.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <random>
#include <vector>

#include "ts_engine.cuh"
#include "ts_segmented.cuh"
#include "ts_transfer.h"

namespace ts {
namespace {

constexpr unsigned long long kHostHugeSegment = 1ull << 22;  // host API: longer segments take the device-wide sort

int width_index(size_t w) { return w == 1 ? 0 : w == 2 ? 1 : w == 4 ? 2 : 3; }

struct SegLayout {
    size_t plan_off, counter_off, lists_off, offs_off, bytes;
    static SegLayout make(size_t n_seg) {
        SegLayout L{};
        L.plan_off = 0;
        L.counter_off = 256;
        L.lists_off = 512;
        L.offs_off = L.lists_off + ((size_t)SEG_NBINS * n_seg * 4 + 255) / 256 * 256;
        L.bytes = L.offs_off + (n_seg + 1) * 8;
        return L;
    }
};

template <typename U, int XF>
__global__ void k_seg_bin_max(const unsigned long long* __restrict__ offsets, size_t n_seg, size_t n,
                              unsigned long long max_len, SegPlan* __restrict__ plan, unsigned int* __restrict__ lists,
                              uint32_t* __restrict__ error) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x; s < n_seg; s += stride) {
        const unsigned long long b = offsets[s], e = offsets[s + 1];
        if (e < b || e > n) {
            atomicOr(error, ERR_BOUNDS);
            continue;
        }
        if (e - b < 2 || e - b > max_len) continue;
        const int bin = seg_bin_of(e - b, SegCfg<U>::CAP);
        const unsigned int i = atomicAdd(&plan->count[bin], 1u);
        lists[(size_t)bin * n_seg + i] = (unsigned int)s;
    }
}

template <typename U, int XF>
ts_status seg_prepare(ts_ctx* c, size_t n, size_t n_seg) {
    ts_status s;
    if ((s = grow(c, c->alt, n * sizeof(U) + 16, "segment scratch")) != TS_OK) return s;
    if ((s = grow(c, c->seg, SegLayout::make(n_seg).bytes, "segment lists")) != TS_OK) return s;
    occupancy_of((const void*)k_seg_sort<U, XF>, SEG_THREADS, MSD_SMEM);
    return TS_OK;
}

template <typename U, int XF>
ts_status seg_enqueue(ts_ctx* c, U* d, size_t n, const unsigned long long* d_off, size_t n_seg,
                      unsigned long long max_len, const SegMethods& m) {
    const SegLayout L = SegLayout::make(n_seg);
    char* base = (char*)c->seg.p;
    SegPlan* plan = (SegPlan*)(base + L.plan_off);
    unsigned int* counter = (unsigned int*)(base + L.counter_off);
    unsigned int* lists = (unsigned int*)(base + L.lists_off);
    mark(c, "segments");
    TS_CUDA(c, cudaMemsetAsync(base, 0, L.lists_off, c->stream));
    const int grid = (int)std::min<size_t>((n_seg + 255) / 256, (size_t)c->sm_count * 8);
    k_seg_bin_max<U, XF><<<std::max(grid, 1), 256, 0, c->stream>>>(d_off, n_seg, n, max_len, plan, lists, c->d_error);
    k_seg_items<<<1, 32, 0, c->stream>>>(plan, m);
    k_seg_sort<U, XF><<<c->sm_count, SEG_THREADS, MSD_SMEM, c->stream>>>(d, d, (U*)c->alt.p, d_off,
                                                                                     lists, n_seg, plan, counter, m);
    c->launches += 3;
    TS_CUDA(c, cudaGetLastError());
    return TS_OK;
}

template <typename U, int XF>
ts_status sort_segments_device(ts_ctx* c, U* d, size_t n, const unsigned long long* d_off, size_t n_seg,
                               unsigned long long max_len) {
    if (n_seg == 0 || n < 2) return TS_OK;
    ts_status s;
    if ((s = seg_prepare<U, XF>(c, n, n_seg)) != TS_OK) return s;
    SegMethods m;
    for (int b = 0; b < SEG_BLOCK_BINS; ++b) m.m[b] = c->seg_methods[width_index(sizeof(U))][b];
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(c->stream, &cs);
    if (!c->use_graphs || c->stream == nullptr || cs != cudaStreamCaptureStatusNone)
        return seg_enqueue<U, XF>(c, d, n, d_off, n_seg, max_len, m);
    // replay the captured launch sequence when nothing it depends on changed
    const size_t key[10] = {sizeof(U) * 4 + (size_t)XF, (size_t)d, n, (size_t)d_off, n_seg, (size_t)max_len,
                            (size_t)c->alt.p, (size_t)c->seg.p,
                            (size_t)(m.m[0] | m.m[1] << 4 | m.m[2] << 8 | m.m[3] << 12), (size_t)c->d_error};
    if (c->seg_graph && std::memcmp(key, c->seg_graph_key, sizeof key) == 0) {
        mark(c, "segments");
        TS_CUDA(c, cudaGraphLaunch(c->seg_graph, c->stream));
        c->launches += 3;
        return TS_OK;
    }
    if (c->seg_graph) {
        cudaGraphExecDestroy(c->seg_graph);
        c->seg_graph = nullptr;
    }
    TS_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    c->capturing = true;
    s = seg_enqueue<U, XF>(c, d, n, d_off, n_seg, max_len, m);
    c->capturing = false;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    if (s != TS_OK) {
        if (g) cudaGraphDestroy(g);
        return s;
    }
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaStreamEndCapture");
    e = cudaGraphInstantiate(&c->seg_graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        c->seg_graph = nullptr;
        return cuda_fail(c, e, "cudaGraphInstantiate");
    }
    std::memcpy(c->seg_graph_key, key, sizeof key);
    mark(c, "segments");
    TS_CUDA(c, cudaGraphLaunch(c->seg_graph, c->stream));
    return TS_OK;
}

// Host segments with the copies overlapped. Segments are independent, so
// the batch goes as transfer_chunks groups of whole segments (about equal
// key counts): group g is sorted as soon as it is on the device, while later
// groups still cross. With a pinned slice each sorted group goes back on a
// stream of its own at once, so copies in and out run together (PCIe carries
// both directions); a pageable slice goes through the staging slots, in
// first and back afterwards, since this thread does those copies itself.
template <typename U, int XF>
ts_status pipeline_segments(ts_ctx* c, U* data, size_t n, const uint64_t* offsets, size_t n_seg,
                            const std::vector<size_t>& huge) {
    const int G = c->transfer_chunks;
    ts_status s;
    if ((s = grow(c, c->keys, n * sizeof(U) + 16, "keys")) != TS_OK) return s;
    if ((s = seg_prepare<U, XF>(c, n, n_seg)) != TS_OK) return s;
    if ((s = pipe_resources(c, (size_t)2 * G + PIPE_SLICES + 2)) != TS_OK) return s;
    U* d = (U*)c->keys.p;
    unsigned long long* d_off = (unsigned long long*)((char*)c->seg.p + SegLayout::make(n_seg).offs_off);
    SegMethods m;
    for (int b = 0; b < SEG_BLOCK_BINS; ++b) m.m[b] = c->seg_methods[width_index(sizeof(U))][b];
    // group g: segments [sg[g], sg[g + 1]), keys [kg[g], kg[g + 1]) (all n keys are copied)
    std::vector<size_t> sg(G + 1), kg(G + 1);
    for (int g = 0; g <= G; ++g) {
        const uint64_t want = offsets[0] + (offsets[n_seg] - offsets[0]) * (uint64_t)g / G;
        sg[g] = g == G ? n_seg : (size_t)(std::lower_bound(offsets, offsets + n_seg, want) - offsets);
        if (g > 0) sg[g] = std::max(sg[g], sg[g - 1]);
        kg[g] = g == 0 ? 0 : g == G ? n : offsets[sg[g]];
    }
    cudaEvent_t* ev = c->pipe_events.data();                    // [G] group g is on the device
    cudaEvent_t* sorted = ev + G + PIPE_SLICES + 2;             // [G] group g is sorted
    Transfer tin(c, data), tout(c, data, c->out_stream);
    TS_CUDA(c, cudaEventRecord(ev[G + PIPE_SLICES], c->stream));
    TS_CUDA(c, cudaStreamWaitEvent(c->copy_stream, ev[G + PIPE_SLICES], 0));
    TS_CUDA(c, cudaStreamWaitEvent(c->out_stream, ev[G + PIPE_SLICES], 0));
    mark(c, "pipeline");
    if ((s = tin.in(d_off, offsets, (n_seg + 1) * 8)) != TS_OK) return s;
    auto copy_in = [&](int g) -> ts_status {
        if (g >= G) return TS_OK;
        ts_status st = tin.in(d + kg[g], data + kg[g], (kg[g + 1] - kg[g]) * sizeof(U));
        if (st != TS_OK) return st;
        TS_CUDA(c, cudaEventRecord(ev[g], c->copy_stream));
        return TS_OK;
    };
    if ((s = copy_in(0)) != TS_OK) return s;
    if ((s = copy_in(1)) != TS_OK) return s;
    size_t next_huge = 0;
    size_t end[64];
    for (int g = 0; g < G; ++g) {
        TS_CUDA(c, cudaStreamWaitEvent(c->stream, ev[g], 0));
        if (sg[g + 1] > sg[g] &&
            (s = seg_enqueue<U, XF>(c, d, n, d_off + sg[g], sg[g + 1] - sg[g], kHostHugeSegment, m)) != TS_OK)
            return s;
        for (; next_huge < huge.size() && huge[next_huge] < sg[g + 1]; ++next_huge) {
            const size_t i = huge[next_huge];
            if ((s = sort_keys_device<U, XF>(c, d + offsets[i], offsets[i + 1] - offsets[i],
                                             (U*)c->alt.p + offsets[i])) != TS_OK)
                return s;
        }
        TS_CUDA(c, cudaEventRecord(sorted[g], c->stream));
        end[g] = kg[g + 1] * sizeof(U);
        if (!tout.pageable && kg[g + 1] > kg[g]) {
            TS_CUDA(c, cudaStreamWaitEvent(c->out_stream, sorted[g], 0));
            TS_CUDA(c, cudaMemcpyAsync(data + kg[g], d + kg[g], (kg[g + 1] - kg[g]) * sizeof(U), cudaMemcpyDeviceToHost,
                                       c->out_stream));
        }
        if ((s = copy_in(g + 2)) != TS_OK) return s;
    }
    mark(c, "end");
    if (tout.pageable) {
        tout.st = c->copy_stream;  // behind every staged copy in
        if ((s = tout.out(data, d, end, sorted, G)) != TS_OK) return s;
    }
    TS_CUDA(c, cudaEventRecord(done_event(c), tout.st));
    TS_CUDA(c, cudaStreamWaitEvent(c->stream, done_event(c), 0));
    return TS_OK;
}

template <typename T, typename U, int XF>
ts_status host_segments(ts_ctx* c, T* data, size_t n, const uint64_t* offsets, size_t n_seg) {
    if (!c) return TS_ERR_INVALID;
    if (n_seg == 0) return TS_OK;
    if (!data || !offsets) return fail(c, TS_ERR_INVALID, "null data or offsets");
    std::vector<size_t> huge;
    for (size_t i = 0; i < n_seg; ++i) {
        if (offsets[i + 1] < offsets[i] || offsets[i + 1] > n)
            return fail(c, TS_ERR_INVALID, "segment offsets must be non-decreasing and end within the slice");
        if (offsets[i + 1] - offsets[i] > kHostHugeSegment) huge.push_back(i);
    }
    if (c->transfer_chunks > 1 && n * sizeof(U) >= c->transfer_min_bytes && n_seg >= 2)
        return pipeline_end(c, pipeline_segments<U, XF>(c, (U*)data, n, offsets, n_seg, huge));
    ts_status s;
    if ((s = grow(c, c->keys, n * sizeof(U) + 16, "keys")) != TS_OK) return s;
    if ((s = seg_prepare<U, XF>(c, n, n_seg)) != TS_OK) return s;
    U* d = (U*)c->keys.p;
    unsigned long long* d_off = (unsigned long long*)((char*)c->seg.p + SegLayout::make(n_seg).offs_off);
    mark(c, "h2d");
    TS_CUDA(c, cudaMemcpyAsync(d, data, n * sizeof(U), cudaMemcpyHostToDevice, c->stream));
    TS_CUDA(c, cudaMemcpyAsync(d_off, offsets, (n_seg + 1) * 8, cudaMemcpyHostToDevice, c->stream));
    if ((s = sort_segments_device<U, XF>(c, d, n, d_off, n_seg, kHostHugeSegment)) != TS_OK) return s;
    for (size_t i : huge)
        if ((s = sort_keys_device<U, XF>(c, d + offsets[i], offsets[i + 1] - offsets[i], (U*)c->alt.p + offsets[i])) !=
            TS_OK)
            return s;
    mark(c, "d2h");
    TS_CUDA(c, cudaMemcpyAsync(data, d, n * sizeof(U), cudaMemcpyDeviceToHost, c->stream));
    return finish(c);
}

// Time each on-chip method on synthetic batches of one length bin and keep
// the fastest, per bin, for keys of this width.
template <typename U>
ts_status autotune(ts_ctx* c) {
    const int lo[SEG_BLOCK_BINS] = {33, 257, 1025, 4097};
    const int hi[SEG_BLOCK_BINS] = {256, 1024, 4096, SegCfg<U>::CAP};
    const size_t target = (size_t)1 << 23;  // keys per timed batch
    std::mt19937_64 rng(0x9E3779B97F4A7C15ull);
    const bool graphs = c->use_graphs;
    c->use_graphs = false;
    const int w = width_index(sizeof(U));
    ts_status s = TS_OK;
    for (int bin = 0; bin < SEG_BLOCK_BINS && s == TS_OK; ++bin) {
        std::vector<uint64_t> offs{0};
        while (offs.back() < target) offs.push_back(offs.back() + lo[bin] + rng() % (uint64_t)(hi[bin] - lo[bin] + 1));
        const size_t n = offs.back(), n_seg = offs.size() - 1;
        std::vector<U> keys(n);
        for (auto& k : keys) k = (U)rng();
        if ((s = grow(c, c->keys, n * sizeof(U) + 16, "tuning keys")) != TS_OK) break;
        if ((s = grow(c, c->gather, 2 * n * sizeof(U) + (n_seg + 1) * 8 + 256, "tuning batch")) != TS_OK) break;
        if ((s = seg_prepare<U, 0>(c, n, n_seg)) != TS_OK) break;
        U* d = (U*)c->keys.p;
        U* master = (U*)c->gather.p;
        unsigned long long* d_off = (unsigned long long*)((char*)c->gather.p + (n * sizeof(U) + 255) / 256 * 256);
        TS_CUDA(c, cudaMemcpyAsync(master, keys.data(), n * sizeof(U), cudaMemcpyHostToDevice, c->stream));
        TS_CUDA(c, cudaMemcpyAsync(d_off, offs.data(), (n_seg + 1) * 8, cudaMemcpyHostToDevice, c->stream));
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        float best = 1e30f;
        int best_m = c->seg_methods[w][bin];
        for (int m = 0; m < SEG_METHODS; ++m) {
            if (!seg_method_ok(bin, m, (int)sizeof(U))) continue;
            c->seg_methods[w][bin] = m;
            float tot = 0.f;
            for (int rep = 0; rep < 4 && s == TS_OK; ++rep) {
                cudaMemcpyAsync(d, master, n * sizeof(U), cudaMemcpyDeviceToDevice, c->stream);
                cudaEventRecord(e0, c->stream);
                s = sort_segments_device<U, 0>(c, d, n, d_off, n_seg, ~0ull);
                cudaEventRecord(e1, c->stream);
                cudaEventSynchronize(e1);
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                if (rep > 0) tot += ms;
            }
            if (tot < best) {
                best = tot;
                best_m = m;
            }
        }
        c->seg_methods[w][bin] = best_m;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    c->use_graphs = graphs;
    if (s != TS_OK) return s;
    return finish(c);
}

}  // namespace
}  // namespace ts

using namespace ts;

extern "C" {

ts_status ts_segments_autotune(ts_ctx* c, size_t key_bytes) {
    if (!c) return TS_ERR_INVALID;
    switch (key_bytes) {
        case 1: return autotune<uint8_t>(c);
        case 2: return autotune<uint16_t>(c);
        case 4: return autotune<uint32_t>(c);
        case 8: return autotune<uint64_t>(c);
    }
    return fail(c, TS_ERR_INVALID, "key_bytes must be 1, 2, 4 or 8");
}

ts_status ts_segments_methods(ts_ctx* c, size_t key_bytes, int* methods, int set) {
    if (!c || !methods || (key_bytes != 1 && key_bytes != 2 && key_bytes != 4 && key_bytes != 8))
        return TS_ERR_INVALID;
    const int w = width_index(key_bytes);
    for (int b = 0; b < SEG_BLOCK_BINS; ++b) {
        if (set) {
            if (!seg_method_ok(b, methods[b], (int)key_bytes))
                return fail(c, TS_ERR_INVALID, "unknown method for this bin and key width");
            c->seg_methods[w][b] = methods[b];
        } else {
            methods[b] = c->seg_methods[w][b];
        }
    }
    return TS_OK;
}

ts_status ts_ctx_use_graphs(ts_ctx* c, int on) {
    if (!c) return TS_ERR_INVALID;
    c->use_graphs = on != 0;
    return TS_OK;
}

#define TS_DEFINE_SEGMENTS(SUF, T, U, XF)                                                                    \
    ts_status ts_sort_segments_##SUF(ts_ctx* c, T* data, size_t n, const uint64_t* offsets, size_t n_seg) {  \
        return host_segments<T, U, XF>(c, data, n, offsets, n_seg);                                        \
    }                                                                                                        \
    ts_status ts_sort_segments_dev_##SUF(ts_ctx* c, T* d_data, size_t n, const uint64_t* d_offsets,          \
                                         size_t n_seg) {                                                     \
        if (!c) return TS_ERR_INVALID;                                                                       \
        if (n_seg && (!d_data || !d_offsets)) return fail(c, TS_ERR_INVALID, "null data or offsets");       \
        return sort_segments_device<U, XF>(c, (U*)d_data, n, (const unsigned long long*)d_offsets, n_seg, ~0ull); \
    }

TS_DEFINE_SEGMENTS(u8, uint8_t, uint8_t, 0)
TS_DEFINE_SEGMENTS(u16, uint16_t, uint16_t, 0)
TS_DEFINE_SEGMENTS(u32, uint32_t, uint32_t, 0)
TS_DEFINE_SEGMENTS(u64, uint64_t, uint64_t, 0)
TS_DEFINE_SEGMENTS(i8, int8_t, uint8_t, 1)
TS_DEFINE_SEGMENTS(i16, int16_t, uint16_t, 1)
TS_DEFINE_SEGMENTS(i32, int32_t, uint32_t, 1)
TS_DEFINE_SEGMENTS(i64, int64_t, uint64_t, 1)
TS_DEFINE_SEGMENTS(f32, float, uint32_t, 2)
TS_DEFINE_SEGMENTS(f64, double, uint64_t, 2)

}  // extern "C"
