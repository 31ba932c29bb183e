/*
 * turbosort.h — C ABI of the B200 radix sort (libturbosort_b200.so).
 *
 * Drop-in for the sort path of the turbosort crate (Rust, 0.2.2). Each entry
 * point names the crate function it replaces (file:line in the crate). The
 * crate's generic functions over its ten SortableKey types (src/key.rs:64-77)
 * become one symbol per type, suffixed u8 u16 u32 u64 i8 i16 i32 i64 f32 f64,
 * which is what an `extern "C"` binding per type would call. Floats sort in
 * total_cmp order (src/key.rs:162-197): -NaN < -inf < ... < -0.0 < +0.0 < ...
 * < +inf < +NaN, and every bit pattern comes back unchanged.
 *
 * Host entry points take host slices, as the crate does: they copy to the
 * device, sort there and copy back before returning. `_dev` entry points take
 * device pointers and only enqueue work on the context's stream; call
 * ts_ctx_synchronize() to wait and collect errors.
 *
 * Panics of the crate become status codes: a buffer shorter than the slice
 * (src/dispatch.rs:78-83) is TS_ERR_BUFFER_TOO_SMALL, an apply_order length
 * mismatch (src/by_key.rs:137-141) is TS_ERR_LENGTH_MISMATCH. A context is
 * used by one host thread at a time.
 */
#ifndef TURBOSORT_H
#define TURBOSORT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum ts_status {
    TS_OK = 0,
    TS_ERR_BUFFER_TOO_SMALL = 1, /* src/dispatch.rs:78-83, src/radix/mod.rs:92-97 */
    TS_ERR_LENGTH_MISMATCH = 2,  /* src/by_key.rs:137-141 */
    TS_ERR_CUDA = 3,             /* a CUDA call failed; see ts_ctx_last_error */
    TS_ERR_TIMEOUT = 4,          /* a bounded device wait ran out; the output is not valid */
    TS_ERR_OOM = 5,              /* device memory could not be reserved */
    TS_ERR_INVALID = 6,          /* a null context or pointer, or an unusable argument */
    TS_ERR_NO_DEVICE = 7,        /* no CUDA device */
    TS_ERR_TOO_LARGE = 8,        /* more than u32::MAX elements where positions are u32 */
    TS_ERR_INTERNAL = 9          /* a device-side bounds check fired */
} ts_status;

typedef struct ts_ctx ts_ctx;

/* Context: a CUDA stream plus device scratch that grows to the largest sort
 * (like SortByKeyBuffer, src/by_key.rs:40-90) and is kept between calls. */
ts_status ts_ctx_create(int device, ts_ctx **out);
void ts_ctx_destroy(ts_ctx *ctx);
/* Use `stream` (a cudaStream_t, or NULL for the legacy default stream)
 * instead of the context's own stream. */
ts_status ts_ctx_set_stream(ts_ctx *ctx, void *stream);
void *ts_ctx_stream(ts_ctx *ctx);
/* Wait for the context's stream; reports errors raised by kernels. */
ts_status ts_ctx_synchronize(ts_ctx *ctx);
/* Reserve scratch for `n` elements of `key_bytes`, with positions when
 * `with_order` (SortByKeyBuffer::with_capacity, src/by_key.rs:74-81). */
ts_status ts_ctx_reserve(ts_ctx *ctx, size_t n, size_t key_bytes, int with_order);
/* Elements of `key_bytes` the context can sort without growing
 * (SortByKeyBuffer::capacity, src/by_key.rs:84-90). */
size_t ts_ctx_capacity(const ts_ctx *ctx, size_t key_bytes, int with_order);
/* Host-slice sorts (ts_sort_<T>, ts_sort_with_buffer_<T>, ts_sort_parallel_<T>,
 * and ts_sort_keys_order_<T> counting keys plus order; keys of 2 bytes or
 * more) of at least `min_bytes` cross PCIe as `chunks` pieces (a power of
 * two, 1 to 64) on a second stream: each piece is sorted (or ordered) while
 * the next one is in flight, the pieces' results are merged pairwise on the
 * device, and the last merge's output is copied back slice by slice while
 * the rest is merged. Host ts_apply_order copies back its gather slice by
 * slice, and host ts_sort_segments_<T> sorts groups of whole segments as
 * they arrive and copies each back at once. A pageable host slice goes through pinned staging
 * slots of the context, filled and emptied by host threads. chunks = 1
 * copies in, sorts and copies out. The output is the same either way.
 * Default: 8 chunks from 64 MiB. */
ts_status ts_ctx_transfer_pipeline(ts_ctx *ctx, int chunks, size_t min_bytes);
const char *ts_ctx_last_error(const ts_ctx *ctx);
const char *ts_status_str(ts_status s);

/* Per-kernel timing with CUDA events on the context's stream (off by default).
 * ts_ctx_timings fills up to `max` (name, total ms, count) triples, sorted by
 * name, and returns how many kernels were seen; it waits for the stream. */
ts_status ts_ctx_enable_timing(ts_ctx *ctx, int on);
int ts_ctx_timings(ts_ctx *ctx, char (*names)[32], double *ms, long *counts, int max);
void ts_ctx_reset_timings(ts_ctx *ctx);
/* Kernels this context has launched so far (all entry points). */
unsigned long long ts_ctx_launches(const ts_ctx *ctx);

/* What the context's last plain sort did (device or host entry point, or a
 * chunk of a host-slice sort); waits for the context's stream. tier: 0 none
 * yet, 1 the small-slice network (n <= 4096), 2 the one-byte counting sort,
 * 3 the LSD passes, 4 the LSD passes in one cooperative launch (2- and
 * 4-byte keys whose tiles fit one wave, up to 1,667,072 keys on a B200). For
 * tiers 3 and 4: mode 0 sorted by passes, 1 input already ascending, 2
 * descending input reversed; passes and pass_digit[] (8-bit
 * digit indices, least significant first) are the scatter passes that ran;
 * divert_shift > 0 means the sort diverted (src/radix/divert.rs:38-81): only
 * the digits from that bit up were sorted by passes, and the runs of keys
 * sharing them were finished directly. */
typedef struct ts_sort_info {
    int32_t tier, mode, passes, divert_shift;
    int32_t pass_digit[16];
    int32_t digit_bits;  /* the LSD's digit width; pass_digit[i] * digit_bits is a pass's shift */
} ts_sort_info;
ts_status ts_ctx_last_sort_info(ts_ctx *ctx, ts_sort_info *info);

/* Diverting of 8-byte keys (on by default, as the crate's sort always
 * diverts when its rule allows, src/radix/mod.rs:240-242). Off, every live
 * digit gets a pass; the output is the same. For comparisons. */
ts_status ts_ctx_set_divert(ts_ctx *ctx, int on);

/* The single-launch LSD (on by default): a keys-only sort of 2- or 4-byte keys
 * whose tiles all fit one wave of CTAs (two an SM) runs every step in one
 * cooperative launch, with bounded grid barriers in place of the look-back.
 * Off, such sorts take the multi-launch LSD; the output is the same. */
ts_status ts_ctx_set_single_launch(ts_ctx *ctx, int on);

/* Test hook for failure detection, no counterpart in the crate: in the next
 * LSD sort on this context (keys or order, more than 4096 keys), the first
 * scatter pass's tile 0 never publishes its look-back entry, and every wait
 * on it gives up after spin_limit rounds (normally about a million); in a
 * single-launch sort, CTA 0 never arrives at the first grid barrier, and
 * every CTA's wait there gives up the same way. The sort then reports
 * TS_ERR_TIMEOUT with every write kept inside the output and scratch
 * buffers; the context stays usable. 0 disarms it. */
ts_status ts_ctx_test_stall_lookback(ts_ctx *ctx, uint32_t spin_limit);

/* The diverting rule of the crate (src/radix/divert.rs:38-54) as the device
 * applies it: how many of the lowest of n_live live digits need no pass, for
 * len keys whose i-th live digit (least significant first) has its largest
 * bucket max_bucket[i]. Host-side, for checks. */
int ts_divert_skippable_digits(int n_live, uint64_t len, const uint64_t *max_bucket);

#define TS_DECLARE_SORTS(SUF, T)                                                                     \
    /* turbosort::sort (src/lib.rs:99): ascending, in place. */                                       \
    ts_status ts_sort_##SUF(ts_ctx *ctx, T *data, size_t n);                                          \
    /* turbosort::sort_with_buffer (src/lib.rs:122): the buffer must hold n elements. */              \
    ts_status ts_sort_with_buffer_##SUF(ts_ctx *ctx, T *data, size_t n, T *buf, size_t buf_len);      \
    /* turbosort::sort_parallel (src/lib.rs:224): the same device sort. */                            \
    ts_status ts_sort_parallel_##SUF(ts_ctx *ctx, T *data, size_t n);                                 \
    /* sort_by_key_with_buffer + SortByKeyBuffer::order (src/by_key.rs:175-233, :108): the keys the   \
     * closure returned, one per element; writes order[i] = source index of output slot i (stable).   \
     * Returns TS_ERR_TOO_LARGE above u32::MAX elements, where the crate leaves order() empty. */      \
    ts_status ts_sort_keys_order_##SUF(ts_ctx *ctx, const T *keys, size_t n, uint32_t *order);        \
    /* Device-resident forms; enqueued on the context's stream. */                                    \
    ts_status ts_sort_dev_##SUF(ts_ctx *ctx, T *d_data, size_t n);                                    \
    ts_status ts_sort_dev_with_buffer_##SUF(ts_ctx *ctx, T *d_data, size_t n, T *d_buf, size_t buf_len); \
    ts_status ts_sort_keys_order_dev_##SUF(ts_ctx *ctx, const T *d_keys, size_t n, uint32_t *d_order);

TS_DECLARE_SORTS(u8, uint8_t)
TS_DECLARE_SORTS(u16, uint16_t)
TS_DECLARE_SORTS(u32, uint32_t)
TS_DECLARE_SORTS(u64, uint64_t)
TS_DECLARE_SORTS(i8, int8_t)
TS_DECLARE_SORTS(i16, int16_t)
TS_DECLARE_SORTS(i32, int32_t)
TS_DECLARE_SORTS(i64, int64_t)
TS_DECLARE_SORTS(f32, float)
TS_DECLARE_SORTS(f64, double)

/* SortByKeyBuffer::apply_order (src/by_key.rs:136-144, :315-334): position i of
 * `data` (n elements of `elem_size` bytes) gets the element that was at
 * order[i]. `order` must be a permutation of 0..n. */
ts_status ts_apply_order(ts_ctx *ctx, void *data, size_t n, size_t elem_size, const uint32_t *order,
                         size_t order_len);
ts_status ts_apply_order_dev(ts_ctx *ctx, void *d_data, size_t n, size_t elem_size, const uint32_t *d_order,
                             size_t order_len);

/* Segmented batch sort (no single counterpart in the crate: the crate sorts
 * each slice with its own `sort` call, src/lib.rs:99, as its small_batches
 * benchmark does, benches/sort_bench.rs:229-250). Sorts every segment
 * data[offsets[i] .. offsets[i+1]) in place, independently, for i < n_seg;
 * offsets holds n_seg + 1 non-decreasing entries ending within n. One device
 * launch sorts the whole batch: segments are binned by length (32 keys and
 * fewer: a warp each; up to 16384 (8192 for 8-byte keys): on chip; longer: a
 * CTA each, by one MSD pass in shared memory up to 49.6K 4-byte or 24.8K
 * 8-byte keys, else by an LSD through L2; host calls send segments above 2^22
 * keys to the device-wide sort). The _dev
 * form replays a captured CUDA graph when called again with the same
 * pointers and sizes. Segments must hold fewer than 2^31 keys. */
#define TS_DECLARE_SEGMENTS(SUF, T)                                                                       \
    ts_status ts_sort_segments_##SUF(ts_ctx *ctx, T *data, size_t n, const uint64_t *offsets, size_t n_seg); \
    ts_status ts_sort_segments_dev_##SUF(ts_ctx *ctx, T *d_data, size_t n, const uint64_t *d_offsets, size_t n_seg);

TS_DECLARE_SEGMENTS(u8, uint8_t)
TS_DECLARE_SEGMENTS(u16, uint16_t)
TS_DECLARE_SEGMENTS(u32, uint32_t)
TS_DECLARE_SEGMENTS(u64, uint64_t)
TS_DECLARE_SEGMENTS(i8, int8_t)
TS_DECLARE_SEGMENTS(i16, int16_t)
TS_DECLARE_SEGMENTS(i32, int32_t)
TS_DECLARE_SEGMENTS(i64, int64_t)
TS_DECLARE_SEGMENTS(f32, float)
TS_DECLARE_SEGMENTS(f64, double)

/* The on-chip method of each segment length bin (32,256] (256,1024]
 * (1024,4096] (4096,16384 or 8192], per key width: 0 bitonic network, 1 radix with
 * 4-bit digits, 2 radix with 8-bit digits, 3 one MSD pass over the key range
 * in shared memory then each key ranked inside its short sub-range, 4 (first
 * bin only) one warp a segment, eight keys a lane in registers, 5 (second bin,
 * keys of up to 4 bytes) one warp a segment, 16 or 32 keys a lane, 6 (third and
 * fourth bins, keys of 4 and 8 bytes) the MSD pass by thread groups, four or
 * two segments a CTA at once. ts_segments_autotune times every
 * method on synthetic batches of each bin on this GPU and keeps the fastest;
 * ts_segments_methods reads (set = 0) or sets (set = 1) the four methods. */
ts_status ts_segments_autotune(ts_ctx *ctx, size_t key_bytes);
ts_status ts_segments_methods(ts_ctx *ctx, size_t key_bytes, int *methods, int set);
/* The plain LSD's autotuner (no counterpart in the crate, whose digit widths
 * and thresholds are compile-time constants measured on its author's CPUs,
 * src/radix/mod.rs:38-54). Each onesweep tile variant (keys a thread: 22, 11,
 * 5 for 4-byte keys; 11, 5, 2 for 8-byte; 32, 16, 8 for 2-byte; 8-bit digits)
 * and the 9-, 10- and 11-bit digit widths are timed on random keys of one
 * length per length bin (n < 2^22, n < 2^25, larger) and the fastest is kept
 * per key width and bin; ms, if not null, receives the 3 x 6 median times
 * (bin-major: the three 8-bit variants, then 9, 10 and 11 bits).
 * ts_lsd_variants reads (set = 0) or sets (set = 1) the three variants of a
 * key width; ts_lsd_variant_ipt gives a variant's keys a thread.
 * ts_lsd_digit_bits reads or sets the digit width per length bin, 4..11 bits
 * (the crate sorts with 8-bit digits and, for long u64 slices, 11-bit ones,
 * src/radix/mod.rs:43-54); widths other than 8 apply to keys-only sorts of
 * fewer than 2^31 keys and never divert. */
ts_status ts_lsd_autotune(ts_ctx *ctx, size_t key_bytes, float *ms);
ts_status ts_lsd_variants(ts_ctx *ctx, size_t key_bytes, int *variants, int set);
int ts_lsd_variant_ipt(size_t key_bytes, int variant);
ts_status ts_lsd_digit_bits(ts_ctx *ctx, size_t key_bytes, int *bits, int set);
/* The tuning cache: the LSD variants and digit widths and the segmented
 * sort's methods of every key width, in a JSON file keyed by the GPU's name. _load leaves the context
 * as it is when the file is missing or was written on another GPU, and sets
 * *loaded to 1 when it took the file's choices. */
ts_status ts_ctx_tune_save(ts_ctx *ctx, const char *path);
ts_status ts_ctx_tune_load(ts_ctx *ctx, const char *path, int *loaded);
/* Capture and replay CUDA graphs for repeated segmented sorts (on by default). */
ts_status ts_ctx_use_graphs(ts_ctx *ctx, int on);

/* Learned-partition sort (no counterpart in the crate; its output equals
 * ts_sort_<T>, i.e. the crate's sort, src/dispatch.rs:31). A 1-in-sample_every
 * sample of the keys is ranked by the plain radix sort. A two-level
 * piecewise-linear CDF model is fitted to it on the GPU: the root puts
 * `leaves` + 1 knots at the sample's quantiles and picks a key's leaf; each
 * leaf is an 8-piece linear CDF over its own key range whose heights
 * train_iters Adam steps fit to the sample's ranks (hand-written forward and
 * backward kernels, FP32). One partition pass puts every key in one of
 * 2^buckets_log2 buckets through the model, whose bucket map is
 * non-decreasing in the key by construction; one segmented launch sorts every
 * bucket. When the largest bucket exceeds overflow_factor x the mean, or the
 * model's largest CDF error on the sample exceeds max_cdf_error, the keys take
 * the plain sort instead (stats->fell_back = 1). use_model = 0 keeps the same
 * partition with equal-width buckets over the key range and no model (the
 * ablation); train_iters = 0 keeps the untrained leaves (linear in the key). */
typedef struct ts_learned_params {
    uint32_t buckets_log2;   /* 12..15 */
    uint32_t sample_every;   /* sample 1 key in this many */
    uint32_t leaves;         /* 2..2048 (with the buckets, within shared memory) */
    uint32_t train_iters;    /* Adam steps */
    float lr;                /* Adam step size, as a fraction of each leaf's initial RMS rank error */
    float overflow_factor;   /* fallback when max bucket > this x mean */
    float max_cdf_error;     /* fallback when the sample's max |CDF error| exceeds this */
    int32_t use_model;       /* 0: equal-width buckets (ablation) */
    uint64_t corrupt_seed;   /* test hook, 0 = off: overwrite the trained leaves with
                                arbitrary values before the partition (output stays exact) */
    uint32_t route_passes;   /* cost route (default 4): when the plain sort would need at most
                                this many scatter passes (estimated from the sample's digit
                                histograms, diverting included; keys of at most this many bytes
                                need no estimate), the plain sort runs instead (reason 4);
                                0 = never */
    int32_t verify;          /* 1 = sort a copy with the plain LSD as well and count
                                the keys where the outputs differ (stats->verify_mismatches);
                                any difference returns TS_ERR_INTERNAL */
} ts_learned_params;

typedef struct ts_learned_stats {
    uint64_t n, sample_size, buckets, max_bucket;
    double mean_bucket, imbalance;           /* imbalance = max_bucket / mean_bucket */
    double train_loss_first, train_loss_last;  /* sample MSE before the first and after the last step */
    float max_cdf_error;
    uint32_t train_iters;
    int32_t fell_back;  /* 1: the plain sort produced the output */
    int32_t reason;     /* 1 bucket overflow, 2 CDF error, 3 input below 2^20 keys,
                           4 routed: the plain sort's estimated passes <= route_passes */
    float ms_sample, ms_train, ms_partition, ms_buckets;
    int32_t est_plain_passes;     /* the plain sort's estimated scatter passes (-1: not estimated) */
    int32_t verified;             /* 1: the verify pass compared the output with the plain sort's */
    uint64_t verify_mismatches;   /* keys where they differ (0 when correct) */
    float ms_verify;
    float pad;
} ts_learned_stats;

void ts_learned_defaults(ts_learned_params *params);

#define TS_DECLARE_LEARNED(SUF, T)                                                                    \
    ts_status ts_sort_learned_##SUF(ts_ctx *ctx, T *data, size_t n, const ts_learned_params *params,   \
                                    ts_learned_stats *stats);                                           \
    ts_status ts_sort_learned_dev_##SUF(ts_ctx *ctx, T *d_data, size_t n, const ts_learned_params *params, \
                                        ts_learned_stats *stats);

TS_DECLARE_LEARNED(u32, uint32_t)
TS_DECLARE_LEARNED(u64, uint64_t)
TS_DECLARE_LEARNED(i32, int32_t)
TS_DECLARE_LEARNED(i64, int64_t)
TS_DECLARE_LEARNED(f32, float)
TS_DECLARE_LEARNED(f64, double)

/* The learned leaves' gradient on device arrays, for checking the backward
 * kernel. Leaf j (of `leaves`) owns samples first[j]..last[j] (-1: none) of
 * t[] (position in the leaf, [0, 1]) and y[] (target CDF value); its 8-piece
 * linear CDF has interior breakpoints bp[7j .. 7j+6] and heights
 * v[9j .. 9j+8], so prediction_i = y0[j] + h[j] * PL_j(t_i). Writes
 * grad[9j + q] = dL/dv[9j + q] of the mean squared error
 * L = (1/m) sum_i (prediction_i - y_i)^2, and L to *loss. A leaf whose range is
 * not within 0..m-1 counts as empty. */
ts_status ts_lm_gradients(ts_ctx *ctx, const float *d_t, const float *d_y, size_t m, int leaves, const int *d_first,
                          const int *d_last, const float *d_bp, const float *d_y0, const float *d_h, const float *d_v,
                          float *d_grad, double *loss);

/* No counterpart in the reference. The device sort of u32 keys for callers
 * that cannot allocate device memory: those whose framework owns all device
 * memory and forbids raw cudaMalloc, those on latency-critical paths where an
 * allocation's implicit synchronisation would stall other streams, and those
 * held to a memory budget fixed at start-up. It needs no context and calls no
 * allocating routine: its scratch is one fixed device array inside the library
 * (about 18 MB, held by every GPU that loads the library until exit), so it
 * sorts at most TS_NOALLOC_MAX_KEYS keys and returns TS_ERR_TOO_LARGE above
 * that. The sort runs on `stream` (a cudaStream_t, or NULL for the legacy
 * default stream) and the call returns when it is done. The first call on a
 * device looks up the array's address there; make that first call before any
 * stream capture. Each process has one such array per device, shared by all
 * of that process's calls on the device; they would race if they overlapped on
 * the GPU, so the library runs them one at a time (each call blocks until its
 * sort is done, also when it returns an error). Not for use across
 * cudaDeviceReset, which discards the library's device code and the array. */
#define TS_NOALLOC_MAX_KEYS ((size_t)1 << 22)
ts_status ts_sort_dev_noalloc_u32(uint32_t *d_data, size_t n, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* TURBOSORT_H */
