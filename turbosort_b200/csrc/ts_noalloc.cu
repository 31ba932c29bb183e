// ts_noalloc.cu — ts_sort_dev_noalloc_u32: the device sort of u32 keys
// without any device allocation.
//
// Some callers cannot call cudaMalloc: code inside a framework that owns all
// device memory through its own allocator and forbids raw allocations,
// code on a latency-critical path where an allocation's implicit device
// synchronisation would stall other streams, and code that runs under a
// memory budget fixed at start-up. This entry point serves them: every
// buffer the sort needs beyond the caller's keys (the ping-pong copy of the
// keys, the look-back array, histograms, scans, counters and the error word)
// lives in one file-scope device array of fixed size, loaded with the
// library and held by every GPU that loads it until the process exits.
//
// Each process has its own copy of the array on each device, shared by every
// call that process makes on that device; it keeps the last call's contents,
// and the sort clears what must start at zero (histograms, counters, the
// look-back region, the error word) on the caller's stream before using it.
// Calls would race on the array if they overlapped on the GPU, so calls in
// one process are serialised here (a lock held until the call's work has
// finished on the GPU, on success and on every error return alike).
// The array's device address is looked up once per device; after
// cudaDeviceReset the library's device code and the array are gone, so the
// entry point must not be used across a reset.
#include <cuda_runtime.h>

#include <mutex>

#include "ts_engine.cuh"

namespace {

using Cfg = ts::LsdCfg<uint32_t, false>;

constexpr size_t kMaxKeys = TS_NOALLOC_MAX_KEYS;
constexpr size_t kTiles = (kMaxKeys + Cfg::TILE - 1) / Cfg::TILE;
constexpr size_t kAltBytes = kMaxKeys * 4;
constexpr size_t kLookbackBytes = 2 * kTiles * Cfg::RADIX * 4;
constexpr size_t kMetaBytes = 64 * 1024;  // scan state, plan, counters, histograms, scans, carries
constexpr size_t kErrorBytes = 256;
constexpr size_t kScratchBytes = kAltBytes + kLookbackBytes + kMetaBytes + kErrorBytes;

// The scratch. In host code this name is only a stand-in for the device
// array; its device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
ts_ctx* g_ctx[kMaxDevices] = {};

// Once per device, with that device current: a context whose buffers are
// carved out of the scratch array, with capacities that never need growing.
ts_status setup(int device, ts_ctx** out) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (g_ctx[device]) {
        *out = g_ctx[device];
        return TS_OK;
    }
    unsigned char* base = nullptr;
    if (cudaGetSymbolAddress((void**)&base, g_scratch) != cudaSuccess || !base) {
        cudaGetLastError();
        return TS_ERR_CUDA;
    }
    const ts::MetaLayout m = ts::MetaLayout::make(Cfg::ND, Cfg::RADIX, Cfg::ND);
    if (m.bytes > kMetaBytes) return TS_ERR_INTERNAL;
    ts_ctx* c = new ts_ctx();
    c->device = device;
    if (cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
        cudaGetLastError();
        delete c;
        return TS_ERR_CUDA;
    }
    c->own_stream = false;
    c->use_graphs = false;  // instantiating a graph could allocate
    // the scratch is sized for the largest tiles (fewest look-back entries)
    for (auto& row : c->lsd_variant)
        for (int& v : row) v = 0;
    c->coop = false;  // the multi-launch LSD, whose metadata fits the scratch
    c->alt.p = base;
    c->alt.cap = kAltBytes;
    c->lookback.p = base + kAltBytes;
    c->lookback.cap = kLookbackBytes;
    c->meta.p = base + kAltBytes + kLookbackBytes;
    c->meta.cap = kMetaBytes;
    c->d_error = reinterpret_cast<uint32_t*>(base + kAltBytes + kLookbackBytes + kMetaBytes);
    g_ctx[device] = c;
    *out = c;
    return TS_OK;
}

}  // namespace

extern "C" ts_status ts_sort_dev_noalloc_u32(uint32_t* d_data, size_t n, void* stream) {
    if (n > kMaxKeys) return TS_ERR_TOO_LARGE;
    if (n <= 1) return TS_OK;
    if (!d_data) return TS_ERR_INVALID;
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices) {
        cudaGetLastError();
        return TS_ERR_CUDA;
    }
    ts_ctx* c = nullptr;
    ts_status s = setup(device, &c);
    if (s != TS_OK) return s;
    std::lock_guard<std::mutex> lock(g_mu);  // one call at a time per process
    c->stream = (cudaStream_t)stream;
    // on an error after the first enqueue, wait for what was queued before
    // the lock is released: the next call must not meet it on the array
    auto drain = [&](ts_status st) {
        cudaStreamSynchronize(c->stream);
        cudaGetLastError();
        return st;
    };
    if (cudaMemsetAsync(c->d_error, 0, 4, c->stream) != cudaSuccess) {
        cudaGetLastError();
        return drain(TS_ERR_CUDA);
    }
    s = ts::sort_keys_device<uint32_t, 0>(c, d_data, n, nullptr);
    if (s != TS_OK) return drain(s);
    uint32_t err = 0;
    if (cudaMemcpyAsync(&err, c->d_error, 4, cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
        cudaStreamSynchronize(c->stream) != cudaSuccess) {
        cudaGetLastError();
        return drain(TS_ERR_CUDA);
    }
    if (err & ts::ERR_TIMEOUT) return TS_ERR_TIMEOUT;
    if (err & ts::ERR_BOUNDS) return TS_ERR_INTERNAL;
    return TS_OK;
}
