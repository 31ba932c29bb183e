// ts_tune.cu — the autotuner of the plain LSD and the tuning cache.
//
// ts_lsd_autotune times every tile variant of the 8-bit onesweep pass (keys a
// thread 22/11/5 for 4-byte keys, 11/5/2 for 8-byte, 32/16/8 for 2-byte) and
// the 9-, 10- and 11-bit digit widths on device-made random keys of one
// length per length bin, and keeps the fastest per key width and bin in the
// context. Widths below 8 bits are not timed: on full-width keys they never
// need fewer passes than bytes do (ts_lsd_digit_bits still sets them). ts_ctx_tune_save / _load keep those
// choices, and the segmented sort's per-bin methods, in a JSON file keyed by
// the GPU's name, so a process can skip the measurement on a GPU it has
// tuned before.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "ts_engine.cuh"
#include "ts_segmented.cuh"

namespace ts {
namespace {

template <typename U>
__global__ void k_tune_keys(U* d, size_t n, unsigned long long seed) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        unsigned long long x = (i + 1) * 0x9E3779B97F4A7C15ull ^ seed;  // splitmix64 finaliser
        x ^= x >> 30;
        x *= 0xBF58476D1CE4E5B9ull;
        x ^= x >> 27;
        x *= 0x94D049BB133111EBull;
        x ^= x >> 31;
        d[i] = (U)x;
    }
}

// timed per length bin: the 8-bit tile variants, then 9-, 10- and 11-bit digits
constexpr int LSD_TUNE_CANDIDATES = LSD_VARIANTS + 3;

// the representative length of each bin
size_t bin_length(int bin, size_t key_bytes) {
    if (bin == 0) return (size_t)1 << 20;
    if (bin == 1) return (size_t)1 << 23;
    return key_bytes == 8 ? (size_t)1 << 26 : (size_t)1 << 27;
}

template <typename U>
ts_status tune(ts_ctx* c, float* ms_out) {
    const int w = width_slot(sizeof(U));
    // the variants serve the multi-launch LSD: single-launch sorts (short
    // slices) are left out of the timing
    const bool graphs = c->use_graphs, coop = c->coop;
    c->use_graphs = false;
    c->coop = false;
    ts_status s = TS_OK;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (int bin = 0; bin < LSD_BINS && s == TS_OK; ++bin) {
        const size_t n = bin_length(bin, sizeof(U));
        if ((s = grow(c, c->gather, 2 * n * sizeof(U) + 256, "tuning keys")) != TS_OK) break;
        U* master = (U*)c->gather.p;
        U* d = (U*)((char*)c->gather.p + (n * sizeof(U) + 255) / 256 * 256);
        k_tune_keys<U><<<c->sm_count * 4, 256, 0, c->stream>>>(master, n, 0x243F6A8885A308D3ull + bin);
        float best = 1e30f;
        int best_v = c->lsd_variant[w][bin], best_b = c->lsd_bits[w][bin];
        // candidates: the 8-bit tile variants, then the wider digits (their own tile)
        for (int v = 0; v < LSD_TUNE_CANDIDATES && s == TS_OK; ++v) {
            const int cand_v = v < LSD_VARIANTS ? v : 0;
            const int cand_b = v < LSD_VARIANTS ? 8 : 8 + (v - LSD_VARIANTS + 1);
            c->lsd_variant[w][bin] = cand_v;
            c->lsd_bits[w][bin] = cand_b;
            std::vector<float> t;
            for (int rep = 0; rep < 6 && s == TS_OK; ++rep) {
                cudaMemcpyAsync(d, master, n * sizeof(U), cudaMemcpyDeviceToDevice, c->stream);
                cudaEventRecord(e0, c->stream);
                s = sort_keys_device<U, 0>(c, d, n, nullptr);
                cudaEventRecord(e1, c->stream);
                cudaEventSynchronize(e1);
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                if (rep > 0) t.push_back(ms);
            }
            if (t.empty()) break;
            std::sort(t.begin(), t.end());
            const float med = t[t.size() / 2];
            if (ms_out) ms_out[bin * LSD_TUNE_CANDIDATES + v] = med;
            if (med < best) {
                best = med;
                best_v = cand_v;
                best_b = cand_b;
            }
        }
        c->lsd_variant[w][bin] = best_v;
        c->lsd_bits[w][bin] = best_b;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->use_graphs = graphs;
    c->coop = coop;
    if (s != TS_OK) return s;
    return finish(c);
}

std::string gpu_name(int device) {
    cudaDeviceProp p{};
    if (cudaGetDeviceProperties(&p, device) != cudaSuccess) {
        cudaGetLastError();
        return "unknown";
    }
    std::string s(p.name);
    for (char& ch : s)
        if (ch == '"' || ch == '\\') ch = '_';
    return s;
}

// the integers of the JSON array that follows `"<key>": ` after `from`
bool read_array(const std::string& t, size_t from, const std::string& key, int* out, int count) {
    const size_t k = t.find("\"" + key + "\"", from);
    if (k == std::string::npos) return false;
    size_t i = t.find('[', k);
    if (i == std::string::npos) return false;
    ++i;
    for (int j = 0; j < count; ++j) {
        while (i < t.size() && (t[i] == ' ' || t[i] == ',' || t[i] == '\n')) ++i;
        char* end = nullptr;
        const long v = std::strtol(t.c_str() + i, &end, 10);
        if (end == t.c_str() + i) return false;
        out[j] = (int)v;
        i = (size_t)(end - t.c_str());
    }
    return true;
}

}  // namespace
}  // namespace ts

using namespace ts;

extern "C" {

ts_status ts_lsd_autotune(ts_ctx* c, size_t key_bytes, float* ms) {
    if (!c) return TS_ERR_INVALID;
    switch (key_bytes) {
        case 2: return tune<uint16_t>(c, ms);
        case 4: return tune<uint32_t>(c, ms);
        case 8: return tune<uint64_t>(c, ms);
    }
    return fail(c, TS_ERR_INVALID, "the plain LSD is tuned for key_bytes 2, 4 or 8");
}

ts_status ts_lsd_variants(ts_ctx* c, size_t key_bytes, int* variants, int set) {
    if (!c || !variants || (key_bytes != 2 && key_bytes != 4 && key_bytes != 8)) return TS_ERR_INVALID;
    const int w = width_slot(key_bytes);
    for (int b = 0; b < LSD_BINS; ++b) {
        if (set) {
            if (variants[b] < 0 || variants[b] >= LSD_VARIANTS) return fail(c, TS_ERR_INVALID, "unknown variant");
        } else {
            variants[b] = c->lsd_variant[w][b];
        }
    }
    if (set)
        for (int b = 0; b < LSD_BINS; ++b) c->lsd_variant[w][b] = variants[b];
    return TS_OK;
}

ts_status ts_lsd_digit_bits(ts_ctx* c, size_t key_bytes, int* bits, int set) {
    if (!c || !bits || (key_bytes != 2 && key_bytes != 4 && key_bytes != 8)) return TS_ERR_INVALID;
    const int w = width_slot(key_bytes);
    for (int b = 0; b < LSD_BINS; ++b) {
        if (set) {
            if (bits[b] < LSD_MIN_BITS || bits[b] > LSD_MAX_BITS)
                return fail(c, TS_ERR_INVALID, "digit width outside 4..11 bits");
        } else {
            bits[b] = c->lsd_bits[w][b];
        }
    }
    if (set)
        for (int b = 0; b < LSD_BINS; ++b) c->lsd_bits[w][b] = bits[b];
    return TS_OK;
}

int ts_lsd_variant_ipt(size_t key_bytes, int variant) {
    if (variant < 0 || variant >= LSD_VARIANTS) return 0;
    switch (key_bytes) {
        case 2: return LsdCfg<uint16_t, false>::IPT0 >> variant;
        case 4: return LsdCfg<uint32_t, false>::IPT0 >> variant;
        case 8: return LsdCfg<uint64_t, false>::IPT0 >> variant;
    }
    return 0;
}

ts_status ts_ctx_tune_save(ts_ctx* c, const char* path) {
    if (!c || !path) return TS_ERR_INVALID;
    FILE* f = std::fopen(path, "w");
    if (!f) return fail(c, TS_ERR_INVALID, std::string("cannot write ") + path);
    std::fprintf(f, "{\n  \"gpu\": \"%s\",\n  \"sm_count\": %d,\n  \"lsd_bins\": [\"n < 2^22\", \"n < 2^25\", \"larger\"],\n",
                 gpu_name(c->device).c_str(), c->sm_count);
    std::fprintf(f, "  \"lsd\": {");
    const int wb[3] = {2, 4, 8};
    for (int i = 0; i < 3; ++i) {
        const int w = width_slot((size_t)wb[i]);
        std::fprintf(f, "%s\"%d\": [%d, %d, %d]", i ? ", " : "", wb[i], c->lsd_variant[w][0], c->lsd_variant[w][1],
                     c->lsd_variant[w][2]);
    }
    std::fprintf(f, "},\n  \"segments\": {");
    const int sb[4] = {1, 2, 4, 8};
    for (int i = 0; i < 4; ++i) {
        const int* m = c->seg_methods[i];
        std::fprintf(f, "%s\"%d\": [%d, %d, %d, %d]", i ? ", " : "", sb[i], m[0], m[1], m[2], m[3]);
    }
    std::fprintf(f, "},\n  \"lsd_bits\": {");
    for (int i = 0; i < 3; ++i) {
        const int w = width_slot((size_t)wb[i]);
        std::fprintf(f, "%s\"%d\": [%d, %d, %d]", i ? ", " : "", wb[i], c->lsd_bits[w][0], c->lsd_bits[w][1],
                     c->lsd_bits[w][2]);
    }
    std::fprintf(f, "}\n}\n");
    const bool ok = std::fclose(f) == 0;
    return ok ? TS_OK : fail(c, TS_ERR_INVALID, std::string("cannot write ") + path);
}

ts_status ts_ctx_tune_load(ts_ctx* c, const char* path, int* loaded) {
    if (!c || !path) return TS_ERR_INVALID;
    if (loaded) *loaded = 0;
    FILE* f = std::fopen(path, "r");
    if (!f) return TS_OK;  // nothing tuned yet
    std::string t;
    char buf[4096];
    size_t k;
    while ((k = std::fread(buf, 1, sizeof buf, f)) > 0) t.append(buf, k);
    std::fclose(f);
    const std::string want = "\"gpu\": \"" + gpu_name(c->device) + "\"";
    if (t.find(want) == std::string::npos) return TS_OK;  // tuned on another GPU
    int lsd[3][LSD_BINS], seg[4][4];
    const size_t lp = t.find("\"lsd\":"), sp = t.find("\"segments\":");
    if (lp == std::string::npos || sp == std::string::npos) return fail(c, TS_ERR_INVALID, "malformed tuning file");
    const char* wk[3] = {"2", "4", "8"};
    for (int i = 0; i < 3; ++i)
        if (!read_array(t, lp, wk[i], lsd[i], LSD_BINS)) return fail(c, TS_ERR_INVALID, "malformed tuning file");
    const char* sk[4] = {"1", "2", "4", "8"};
    for (int i = 0; i < 4; ++i)
        if (!read_array(t, sp, sk[i], seg[i], 4)) return fail(c, TS_ERR_INVALID, "malformed tuning file");
    for (auto& row : lsd)
        for (int v : row)
            if (v < 0 || v >= LSD_VARIANTS) return fail(c, TS_ERR_INVALID, "tuning file: unknown variant");
    // digit widths (absent from files written before they were tuned: 8 bits)
    int lbits[3][LSD_BINS];
    for (auto& row : lbits)
        for (int& b : row) b = 8;
    const size_t bp = t.find("\"lsd_bits\":");
    if (bp != std::string::npos)
        for (int i = 0; i < 3; ++i)
            if (!read_array(t, bp, wk[i], lbits[i], LSD_BINS)) return fail(c, TS_ERR_INVALID, "malformed tuning file");
    for (auto& row : lbits)
        for (int b : row)
            if (b < LSD_MIN_BITS || b > LSD_MAX_BITS) return fail(c, TS_ERR_INVALID, "tuning file: digit width");
    const int sbytes[4] = {1, 2, 4, 8};
    for (int i = 0; i < 4; ++i)
        for (int b = 0; b < 4; ++b)
            if (!seg_method_ok(b, seg[i][b], sbytes[i])) return fail(c, TS_ERR_INVALID, "tuning file: unknown method");
    const int wb[3] = {2, 4, 8};
    for (int i = 0; i < 3; ++i)
        for (int b = 0; b < LSD_BINS; ++b) {
            c->lsd_variant[width_slot((size_t)wb[i])][b] = lsd[i][b];
            c->lsd_bits[width_slot((size_t)wb[i])][b] = lbits[i][b];
        }
    for (int i = 0; i < 4; ++i)
        for (int b = 0; b < 4; ++b) c->seg_methods[i][b] = seg[i][b];
    if (loaded) *loaded = 1;
    return TS_OK;
}

}  // extern "C"
