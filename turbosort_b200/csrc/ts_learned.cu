// ts_learned.cu — the learned-partition sort: host orchestration, the
// fallback to the plain LSD, statistics, and the C ABI.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "ts_engine.cuh"
#include "ts_learned.cuh"
#include "ts_transfer.h"
#include "ts_segmented.cuh"

namespace ts {
namespace {

struct Bump {
    char* base;
    size_t off = 0;
    template <typename T>
    T* take(size_t count) {
        off = (off + 255) / 256 * 256;
        T* p = reinterpret_cast<T*>(base + off);
        off += count * sizeof(T);
        return p;
    }
};

struct LmBuffers {
    void* sample;
    LmHead* head;
    LmTables T;
    double* loss;  // [2]: before the first step, after the last
    float* max_err;
    unsigned long long* mismatches;  // the verify pass's count
    unsigned long long *totals, *offsets, *max_bucket, *cur1, *cur2;
    unsigned int *tiles_before, *counter;
    size_t bytes;
};

LmBuffers lm_layout(char* base, size_t m, size_t key_bytes, int leaves, int buckets) {
    Bump b{base};
    LmBuffers B{};
    B.sample = b.take<unsigned char>(m * key_bytes);
    B.head = b.take<LmHead>(1);
    B.T.rootk = b.take<uint32_t>((size_t)1 << lm_depth(leaves));
    B.T.leaf = b.take<LmLeaf>(leaves);
    B.T.bp = b.take<float>((size_t)leaves * (LM_P - 1));
    B.T.c = b.take<float>((size_t)leaves * (LM_P + 1));
    B.T.v = b.take<float>((size_t)leaves * (LM_P + 1));
    B.T.y0 = b.take<float>(leaves);
    B.T.h = b.take<float>(leaves);
    B.T.first = b.take<int>(leaves);
    B.T.last = b.take<int>(leaves);
    B.loss = b.take<double>(2);
    B.max_err = b.take<float>(1);
    B.mismatches = b.take<unsigned long long>(1);
    B.max_bucket = b.take<unsigned long long>(1);
    B.counter = b.take<unsigned int>(1);
    B.totals = b.take<unsigned long long>(buckets);
    B.offsets = b.take<unsigned long long>((size_t)buckets + 1);
    B.cur1 = b.take<unsigned long long>(LM_SUPERS);
    B.cur2 = b.take<unsigned long long>(buckets);
    B.tiles_before = b.take<unsigned int>(LM_SUPERS + 1);
    B.bytes = b.off + 256;
    return B;
}

}  // namespace

// keys where a and b differ
template <typename U>
__global__ void k_lm_compare(const U* __restrict__ a, const U* __restrict__ b, size_t n,
                             unsigned long long* __restrict__ count) {
    unsigned long long c = 0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        c += a[i] != b[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, c);
}

struct Events {
    cudaEvent_t e[7] = {};
    Events() {
        for (auto& x : e) cudaEventCreate(&x);
    }
    ~Events() {
        for (auto& x : e)
            if (x) cudaEventDestroy(x);
    }
    float ms(int a, int b) const {
        float t = 0.f;
        cudaEventElapsedTime(&t, e[a], e[b]);
        return t;
    }
};

template <typename U, int XF>
static ts_status learned_sort_device(ts_ctx* c, U* d, size_t n, const ts_learned_params* P, ts_learned_stats* st) {
    ts_learned_params prm;
    ts_learned_defaults(&prm);
    if (P) prm = *P;
    ts_learned_stats S{};
    S.n = n;
    auto done = [&](ts_status s) {
        if (st) *st = S;
        return s;
    };
    if (n <= 1) return done(TS_OK);
    const int blog = (int)prm.buckets_log2;
    if (blog < 12 || blog > 15) return done(fail(c, TS_ERR_INVALID, "learned partition: buckets_log2 outside 12..15"));
    if (prm.leaves < 2 || prm.leaves > (uint32_t)LM_MAX_LEAVES)
        return done(fail(c, TS_ERR_INVALID, "learned partition: leaves outside 2..2048"));
    const int leaves = (int)prm.leaves;
    const int buckets = 1 << blog;
    const size_t count_smem = lm_smem_bytes(leaves) + (size_t)buckets * 4;
    int max_smem = 0;
    cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
    if (count_smem > (size_t)max_smem)
        return done(fail(c, TS_ERR_INVALID, "learned partition: leaves and buckets exceed shared memory"));
    const size_t every = std::max<uint32_t>(2, prm.sample_every);
    const size_t m = n / every;
    const bool too_small = n < (1u << 20) || m < 2 * (size_t)leaves;  // too small for the model to pay
    const int iters = std::max(0, (int)prm.train_iters);
    S.est_plain_passes = -1;
    if (too_small) {
        S.fell_back = 1;
        S.reason = 3;
        ts_status s3 = sort_keys_device<U, XF>(c, d, n, nullptr);
        if (s3 == TS_OK) s3 = finish(c);
        return done(s3);
    }
    // the cost route: keys of at most route_passes bytes never need more than
    // that many 8-bit passes, so the plain sort runs without a sample
    auto plain = [&](int reason) {
        S.fell_back = 1;
        S.reason = reason;
        ts_status s2 = sort_keys_device<U, XF>(c, d, n, nullptr);
        if (s2 == TS_OK) s2 = finish(c);
        return done(s2);
    };
    if (prm.route_passes > 0 && sizeof(U) <= prm.route_passes) {
        S.est_plain_passes = (int32_t)sizeof(U);
        return plain(4);
    }

    ts_status s;
    LmBuffers B = lm_layout(nullptr, m, sizeof(U), leaves, buckets);
    if ((s = grow(c, c->learn, B.bytes, "learned model")) != TS_OK) return done(s);
    if ((s = grow(c, c->alt, n * sizeof(U) + 16, "partition buffer")) != TS_OK) return done(s);
    if ((s = grow(c, c->gather, n * sizeof(U) + 16, "group buffer")) != TS_OK) return done(s);
    if ((s = grow(c, c->vals0, n * 2 + 16, "bucket ids")) != TS_OK) return done(s);
    if ((s = grow(c, c->vals1, n * 2 + 16, "grouped bucket ids")) != TS_OK) return done(s);
    B = lm_layout((char*)c->learn.p, m, sizeof(U), leaves, buckets);
    unsigned short* ids = (unsigned short*)c->vals0.p;
    unsigned short* ids1 = (unsigned short*)c->vals1.p;
    TS_CUDA(c, cudaFuncSetAttribute((const void*)k_lm_count<U, XF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)count_smem));
    TS_CUDA(c, cudaFuncSetAttribute((const void*)k_lm_split1<U>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)LmSplitSmem<U>::bytes));
    TS_CUDA(c, cudaFuncSetAttribute((const void*)k_lm_split2<U>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)LmSplitSmem<U>::bytes));
    TS_CUDA(c, cudaFuncSetAttribute((const void*)k_lm_finish<U, XF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    MSD_SMEM));

    U* check = nullptr;  // the verify pass's copy of the input
    if (prm.verify) {
        if ((s = grow(c, c->check, n * sizeof(U) + 16, "verify copy")) != TS_OK) return done(s);
        check = (U*)c->check.p;
        TS_CUDA(c, cudaMemcpyAsync(check, d, n * sizeof(U), cudaMemcpyDeviceToDevice, c->stream));
    }

    Events ev;
    mark(c, "lm_sample");
    cudaEventRecord(ev.e[0], c->stream);
    // 1. sample, and its exact ranks from the plain radix sort
    U* sample = (U*)B.sample;
    k_lm_sample<U><<<c->sm_count * 4, 256, 0, c->stream>>>(d, n, every, sample, m, XF);
    ++c->launches;
    if ((s = sort_keys_device<U, 0>(c, sample, m, nullptr)) != TS_OK) return done(s);
    if (prm.route_passes > 0) {
        // the sample's digit histograms stand for the input's: its live
        // digits, and each digit's largest bucket scaled to n keys, give the
        // passes the plain sort would run (diverting included)
        constexpr int ND = (int)sizeof(U);
        unsigned long long maxb[ND];
        const MetaLayout ml = MetaLayout::make(ND, 256, 0);
        TS_CUDA(c, cudaMemcpyAsync(maxb, (const char*)c->meta.p + ml.maxb_off(), sizeof maxb, cudaMemcpyDeviceToHost,
                                   c->stream));
        TS_CUDA(c, cudaStreamSynchronize(c->stream));
        unsigned long long scaled[ND];
        int live = 0;
        for (int dg = 0; dg < ND; ++dg)
            if (maxb[dg]) {
                const double f = (double)maxb[dg] * (double)n / (double)m;
                scaled[live++] = (unsigned long long)std::min<double>((double)n, std::max(1.0, f));
            }
        S.est_plain_passes = live - skippable_digits(live, n, scaled);
        if (S.est_plain_passes <= (int)prm.route_passes) {
            S.ms_sample = 0.f;
            return plain(4);
        }
    }
    mark(c, "lm_fit");
    TS_CUDA(c, cudaMemsetAsync(B.T.first, 0xff, (size_t)leaves * 4, c->stream));
    TS_CUDA(c, cudaMemsetAsync(B.T.last, 0xff, (size_t)leaves * 4, c->stream));
    TS_CUDA(c, cudaMemsetAsync(B.loss, 0, 2 * 8, c->stream));
    TS_CUDA(c, cudaMemsetAsync(B.max_err, 0, 4, c->stream));
    TS_CUDA(c, cudaMemsetAsync(B.max_bucket, 0, 8, c->stream));
    TS_CUDA(c, cudaMemsetAsync(B.counter, 0, 4, c->stream));
    TS_CUDA(c, cudaMemsetAsync(B.totals, 0, (size_t)buckets * 8, c->stream));
    k_lm_root<U><<<1, 1024, 0, c->stream>>>(sample, m, leaves, buckets, prm.use_model ? 1 : 0, B.head, B.T.rootk);
    ++c->launches;
    cudaEventRecord(ev.e[1], c->stream);
    // 2. fit the leaves
    if (prm.use_model) {
        const int grid = c->sm_count * 4;
        k_lm_leaves<U><<<grid, 256, 0, c->stream>>>(sample, m, B.head, B.T.rootk, B.T.first, B.T.last);
        k_lm_init<U><<<(leaves + 255) / 256, 256, 0, c->stream>>>(sample, m, leaves, B.T);
        k_lm_train<U><<<leaves, LM_TRAIN_THREADS, 0, c->stream>>>(sample, m, B.T, iters, prm.lr, B.loss, B.loss + 1,
                                                                  B.max_err);
        c->launches += 3;
        if (prm.corrupt_seed) {
            k_lm_corrupt<<<(leaves + 255) / 256, 256, 0, c->stream>>>(leaves, B.T, prm.corrupt_seed);
            ++c->launches;
        }
        k_lm_bounds<<<1, 1024, 0, c->stream>>>(leaves, buckets, B.T);
        ++c->launches;
    }
    cudaEventRecord(ev.e[2], c->stream);
    // 3. every key's bucket, the bucket sizes and offsets, the largest bucket
    mark(c, "lm_count");
    const int count_grid = std::max<int>(1, std::min<int>(c->sm_count, (int)((n + 4095) / 4096)));
    k_lm_count<U, XF><<<count_grid, 1024, count_smem, c->stream>>>(d, n, B.head, B.T, ids, B.totals);
    k_lm_bucket_scan<<<1, 1024, 0, c->stream>>>(B.totals, buckets, B.offsets, B.max_bucket, B.cur1, B.cur2,
                                               B.tiles_before);
    c->launches += 2;
    TS_CUDA(c, cudaGetLastError());
    // the decision needs these on the host
    double loss[2] = {0, 0};
    float max_err = 0;
    unsigned long long max_bucket = 0;
    TS_CUDA(c, cudaMemcpyAsync(&max_bucket, B.max_bucket, 8, cudaMemcpyDeviceToHost, c->stream));
    TS_CUDA(c, cudaMemcpyAsync(&max_err, B.max_err, 4, cudaMemcpyDeviceToHost, c->stream));
    TS_CUDA(c, cudaMemcpyAsync(loss, B.loss, 16, cudaMemcpyDeviceToHost, c->stream));
    cudaEventRecord(ev.e[3], c->stream);
    TS_CUDA(c, cudaStreamSynchronize(c->stream));
    S.sample_size = m;
    S.buckets = (uint64_t)buckets;
    S.max_bucket = max_bucket;
    S.mean_bucket = (double)n / buckets;
    S.imbalance = (double)max_bucket / S.mean_bucket;
    if (prm.use_model) {
        S.train_loss_first = loss[0];
        S.train_loss_last = loss[1];
        S.max_cdf_error = max_err;
        S.train_iters = (uint32_t)iters;
    }
    S.ms_sample = ev.ms(0, 1);
    S.ms_train = ev.ms(1, 2);
    S.ms_partition = ev.ms(2, 3);
    if ((double)max_bucket > (double)prm.overflow_factor * S.mean_bucket) {
        S.fell_back = 1;
        S.reason = 1;
    } else if (prm.use_model && max_err > prm.max_cdf_error) {
        S.fell_back = 1;
        S.reason = 2;
    }
    if (S.fell_back) {
        cudaEventRecord(ev.e[4], c->stream);
        s = sort_keys_device<U, XF>(c, d, n, nullptr);
        cudaEventRecord(ev.e[5], c->stream);
        if (s == TS_OK) s = finish(c);
        S.ms_buckets = ev.ms(4, 5);
        return done(s);
    }
    // 4. two scatter sweeps (128 groups, then the buckets of each group), then
    // every bucket sorted into d
    U* part = (U*)c->alt.p;
    U* grouped = (U*)c->gather.p;
    const int split_tiles = (int)((n + LM_SPLIT_TILE - 1) / LM_SPLIT_TILE);
    mark(c, "lm_split");
    cudaEventRecord(ev.e[4], c->stream);
    const int split_grid = std::min(split_tiles, 2 * c->sm_count);
    k_lm_split1<U><<<split_grid, LM_SPLIT_THREADS, LmSplitSmem<U>::bytes, c->stream>>>(
        d, ids, n, blog - 7, B.cur1, B.offsets, grouped, ids1, c->d_error);
    k_lm_split2<U><<<2 * c->sm_count, LM_SPLIT_THREADS, LmSplitSmem<U>::bytes, c->stream>>>(
        grouped, ids1, buckets, B.offsets, B.tiles_before, B.cur2, part, c->d_error);
    c->launches += 2;
    mark(c, "lm_finish");
    cudaEventRecord(ev.e[5], c->stream);
    k_lm_finish<U, XF><<<c->sm_count, 1024, MSD_SMEM, c->stream>>>(part, d, grouped, B.offsets, buckets, B.counter);
    ++c->launches;
    TS_CUDA(c, cudaGetLastError());
    cudaEventRecord(ev.e[6], c->stream);
    if (check) {
        // verify: the plain LSD sorts the copy, and the outputs must agree
        // key for key (an exact sort has one output)
        TS_CUDA(c, cudaMemsetAsync(B.mismatches, 0, 8, c->stream));
        if ((s = sort_keys_device<U, XF>(c, check, n, nullptr)) != TS_OK) return done(s);
        k_lm_compare<U><<<c->sm_count * 4, 256, 0, c->stream>>>(d, check, n, B.mismatches);
        ++c->launches;
        TS_CUDA(c, cudaGetLastError());
        cudaEventRecord(ev.e[0], c->stream);
        unsigned long long mism = 0;
        TS_CUDA(c, cudaMemcpyAsync(&mism, B.mismatches, 8, cudaMemcpyDeviceToHost, c->stream));
        s = finish(c);
        S.verified = 1;
        S.verify_mismatches = mism;
        S.ms_verify = ev.ms(6, 0);
        if (s == TS_OK && mism)
            s = fail(c, TS_ERR_INTERNAL, "learned partition: the output differs from the plain sort's");
    } else {
        s = finish(c);
    }
    S.ms_partition += ev.ms(4, 5);
    S.ms_buckets = ev.ms(5, 6);
    return done(s);
}

template <typename U, int XF>
static ts_status staged_learned(ts_ctx* c, Transfer& t, U* data, U* d, size_t n, const ts_learned_params* P,
                                ts_learned_stats* st) {
    cudaEvent_t* ev = c->pipe_events.data();
    ts_status s;
    TS_CUDA(c, cudaEventRecord(ev[0], c->stream));
    TS_CUDA(c, cudaStreamWaitEvent(t.st, ev[0], 0));
    if ((s = t.in(d, data, n * sizeof(U))) != TS_OK) return s;
    TS_CUDA(c, cudaEventRecord(ev[1], t.st));
    TS_CUDA(c, cudaStreamWaitEvent(c->stream, ev[1], 0));
    if ((s = learned_sort_device<U, XF>(c, d, n, P, st)) != TS_OK) return s;
    TS_CUDA(c, cudaEventRecord(slice_events(c)[0], c->stream));
    const size_t end = n * sizeof(U);
    if ((s = t.out(data, d, &end, slice_events(c), 1)) != TS_OK) return s;
    TS_CUDA(c, cudaEventRecord(done_event(c), t.st));
    TS_CUDA(c, cudaStreamWaitEvent(c->stream, done_event(c), 0));
    return TS_OK;
}

template <typename T, typename U, int XF>
static ts_status host_learned(ts_ctx* c, T* data, size_t n, const ts_learned_params* P, ts_learned_stats* st) {
    if (!c) return TS_ERR_INVALID;
    if (n <= 1) return TS_OK;
    if (!data) return fail(c, TS_ERR_INVALID, "null data");
    ts_status s;
    if ((s = grow(c, c->keys, n * sizeof(U) + 16, "keys")) != TS_OK) return s;
    U* d = (U*)c->keys.p;
    if (c->transfer_chunks > 1 && n * sizeof(U) >= c->transfer_min_bytes) {
        // the partition needs every key, so nothing overlaps the copies; a
        // pageable slice still crosses through the staging slots
        if ((s = pipe_resources(c, (size_t)c->transfer_chunks + PIPE_SLICES + 2)) != TS_OK) return s;
        Transfer t(c, data);
        if (t.pageable) return pipeline_end(c, staged_learned<U, XF>(c, t, (U*)data, d, n, P, st));
    }
    TS_CUDA(c, cudaMemcpyAsync(d, data, n * sizeof(U), cudaMemcpyHostToDevice, c->stream));
    if ((s = learned_sort_device<U, XF>(c, d, n, P, st)) != TS_OK) return s;
    TS_CUDA(c, cudaMemcpyAsync(data, d, n * sizeof(U), cudaMemcpyDeviceToHost, c->stream));
    return finish(c);
}

}  // namespace ts

using namespace ts;

extern "C" {

void ts_learned_defaults(ts_learned_params* p) {
    if (!p) return;
    p->buckets_log2 = 14;
    p->sample_every = 100;
    p->leaves = 1024;
    // 2^28 keys on a B200: 8 Adam steps take the Gaussian mixture's largest
    // bucket from 2.76x to 2.38x the mean for 0.1 ms; 32 steps reach 2.35x
    // for 0.43 ms; neither shortens the bucket sorts
    p->train_iters = 8;
    p->lr = 0.5f;
    p->overflow_factor = 4.f;
    p->max_cdf_error = 0.01f;
    p->use_model = 1;
    p->corrupt_seed = 0;
    // measured on a B200 (2^28 keys): the partition (8.8 ms for 8-byte keys)
    // beats the plain sort when that needs five or more 8-byte passes
    // (lognormal f64, diverted to five: 10.6 ms; all eight: 13.0 ms), and
    // loses to four passes of 4-byte keys (7.1 against 4.3 ms)
    p->route_passes = 4;
    p->verify = 0;
}

ts_status ts_lm_gradients(ts_ctx* c, const float* d_t, const float* d_y, size_t m, int leaves, const int* d_first,
                          const int* d_last, const float* d_bp, const float* d_y0, const float* d_h, const float* d_v,
                          float* d_grad, double* loss_out) {
    if (!c) return TS_ERR_INVALID;
    if (!d_t || !d_y || !d_first || !d_last || !d_bp || !d_y0 || !d_h || !d_v || !d_grad || m == 0 || leaves < 1 ||
        leaves > LM_MAX_LEAVES)
        return fail(c, TS_ERR_INVALID, "ts_lm_gradients: null array or unusable size");
    ts_status s;
    if ((s = grow(c, c->meta, 256, "gradient scratch")) != TS_OK) return s;
    double* loss = (double*)c->meta.p;
    LmTables T{};
    T.first = const_cast<int*>(d_first);
    T.last = const_cast<int*>(d_last);
    T.bp = const_cast<float*>(d_bp);
    T.y0 = const_cast<float*>(d_y0);
    T.h = const_cast<float*>(d_h);
    T.v = const_cast<float*>(d_v);
    TS_CUDA(c, cudaMemsetAsync(loss, 0, 8, c->stream));
    TS_CUDA(c, cudaMemsetAsync(d_grad, 0, (size_t)leaves * (LM_P + 1) * 4, c->stream));
    k_lm_grad<<<leaves, LM_TRAIN_THREADS, 0, c->stream>>>(d_t, d_y, m, T, d_grad, loss);
    ++c->launches;
    double l = 0;
    TS_CUDA(c, cudaMemcpyAsync(&l, loss, 8, cudaMemcpyDeviceToHost, c->stream));
    ts_status f = finish(c);
    if (loss_out) *loss_out = l;
    return f;
}

#define TS_DEFINE_LEARNED(SUF, T, U, XF)                                                                      \
    ts_status ts_sort_learned_##SUF(ts_ctx* c, T* data, size_t n, const ts_learned_params* p,                  \
                                    ts_learned_stats* st) {                                                     \
        return host_learned<T, U, XF>(c, data, n, p, st);                                                      \
    }                                                                                                           \
    ts_status ts_sort_learned_dev_##SUF(ts_ctx* c, T* d_data, size_t n, const ts_learned_params* p,            \
                                        ts_learned_stats* st) {                                                 \
        if (!c) return TS_ERR_INVALID;                                                                          \
        if (n > 1 && !d_data) return fail(c, TS_ERR_INVALID, "null data");                                     \
        ts_status s = learned_sort_device<U, XF>(c, (U*)d_data, n, p, st);                                     \
        return s;                                                                                               \
    }

TS_DEFINE_LEARNED(u32, uint32_t, uint32_t, 0)
TS_DEFINE_LEARNED(u64, uint64_t, uint64_t, 0)
TS_DEFINE_LEARNED(i32, int32_t, uint32_t, 1)
TS_DEFINE_LEARNED(i64, int64_t, uint64_t, 1)
TS_DEFINE_LEARNED(f32, float, uint32_t, 2)
TS_DEFINE_LEARNED(f64, double, uint64_t, 2)

}  // extern "C"
