/*
 * turbosort_oracle.c — CPU restatement of the turbosort crate's sort path
 * (ampactor-labs/turbosort 0.2.2, pure Rust).
 *
 * TEST INFRASTRUCTURE ONLY. This is the oracle: tests/, __graft_entry__.smoke()
 * and the CPU-baseline leg of bench.py use it to check and to time the CUDA
 * library. The product never links, loads or calls it.
 *
 * The crate cannot be built in this environment (no Rust toolchain, no
 * network), so this file restates its algorithm in C, step by step, citing the
 * crate's source by file:line. It is pinned against the known-answer vectors
 * of the crate's own tests (tests/golden/, restated there from
 * src/key.rs, src/radix/divert.rs, src/radix/histogram.rs, src/by_key.rs,
 * src/lib.rs, README.md and tests/correctness.rs).
 *
 * Covered:
 *   key transforms          src/key.rs:135-197
 *   sort / sort_with_buffer src/dispatch.rs:31-111, src/presorted.rs:15-65,
 *                           src/radix/mod.rs:61-271,518-600,
 *                           src/radix/histogram.rs:15-110,
 *                           src/radix/prefix_sum.rs:17-24,
 *                           src/radix/scatter.rs:26-221,
 *                           src/radix/divert.rs:38-104
 *   sort_parallel           src/parallel.rs:46-291 (pthreads in place of rayon)
 *   sort_by_key (order)     src/by_key.rs:175-310
 *   apply_order             src/by_key.rs:136-144,315-334
 */
#define _GNU_SOURCE
#include <emmintrin.h>
#include <pthread.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define CAT_(a, b) a##b
#define CAT(a, b) CAT_(a, b)

#define TSO_BUFFER_TOO_SMALL 1

/* Thresholds of the crate. */
enum {
    COUNTING_MIN = 48,         /* dispatch.rs:25 */
    INTERLEAVE_MIN = 8192,     /* histogram.rs:7 */
    WIDE_MIN = 65536,          /* radix/mod.rs:43 */
    MARK_RUNS_MAX = 256,       /* radix/mod.rs:114 */
    LINE_BYTES = 64,           /* scatter.rs:43 */
    COMBINE_MIN = 16384,       /* scatter.rs:202 */
    SLACK_BITS = 2,            /* divert.rs:19 */
    SHORT_RUN = 16,            /* divert.rs:23 */
    MIN_SKIP = 3,              /* divert.rs:28 */
    INSERTION_MAX = 64,        /* by_key.rs:31 */
    SERIAL_SCAN = 4096,        /* parallel.rs:38 */
    PARALLEL_THRESHOLD = 131072 /* parallel.rs:41 */
};
static const size_t STREAM_MIN_BYTES = (size_t)2 << 20; /* scatter.rs:189 */

/* prefix_sum.rs:17-24 */
static void exclusive_prefix_sum(size_t *h, size_t bins) {
    size_t sum = 0;
    for (size_t i = 0; i < bins; i++) {
        size_t c = h[i];
        h[i] = sum;
        sum += c;
    }
}

/* scatter.rs:195-198 — x86_64 streams destinations of 2 MiB and more. */
static int streams_bytes(size_t bytes) { return bytes >= STREAM_MIN_BYTES; }

/* scatter.rs:208-221 — at least 64 non-empty buckets, sizes within ~3%. */
static int wants_combining(const size_t *hist, size_t bins, size_t len) {
    if (len < COMBINE_MIN) return 0;
    size_t buckets = 0, mn = (size_t)-1, mx = 0;
    for (size_t d = 0; d < bins; d++) {
        size_t c = hist[d];
        if (c > 0) {
            buckets++;
            mn = c < mn ? c : mn;
            mx = c > mx ? c : mx;
        }
    }
    return buckets >= 64 && mx - mn <= len / buckets / 32 + 2;
}

/* scatter.rs:157-171 — one 64-byte line with non-temporal stores. */
static inline void stream_line(const void *src, void *dst) {
    const __m128i *s = (const __m128i *)src;
    __m128i *d = (__m128i *)dst;
    _mm_stream_si128(d, _mm_load_si128(s));
    _mm_stream_si128(d + 1, _mm_load_si128(s + 1));
    _mm_stream_si128(d + 2, _mm_load_si128(s + 2));
    _mm_stream_si128(d + 3, _mm_load_si128(s + 3));
}

/* divert.rs:95-104 — log2(x) in eighths of a bit, never above the truth. */
uint32_t tso_log2_eighths(size_t x) {
    uint32_t ip = 63u - (uint32_t)__builtin_clzll((unsigned long long)x);
    size_t frac = ip >= 3 ? (x >> (ip - 3)) & 7 : (x << (3 - ip)) & 7;
    return 8 * ip + (uint32_t)frac;
}

/* divert.rs:38-54 — how many low live digits may be left unsorted. */
size_t tso_skippable_digits(size_t n_live, size_t len, const size_t *max_bucket) {
    if (n_live <= MIN_SKIP) return 0;
    uint32_t log_len = tso_log2_eighths(len);
    uint32_t need = log_len + 8 * SLACK_BITS;
    uint32_t have = 0;
    for (size_t i = n_live; i-- > MIN_SKIP;) {
        have += log_len - tso_log2_eighths(max_bucket[i]);
        if (have >= need) return i;
    }
    return 0;
}

/* Fork-join over `n` tasks on `n` threads (rayon's role in parallel.rs). */
typedef struct {
    void (*fn)(void *, int);
    void *arg;
    int t;
} thread_job;
static void *thread_main(void *p) {
    thread_job *j = p;
    j->fn(j->arg, j->t);
    return NULL;
}
static void run_threads(int n, void (*fn)(void *, int), void *arg) {
    if (n <= 1) {
        if (n == 1) fn(arg, 0);
        return;
    }
    pthread_t *th = malloc(sizeof(pthread_t) * (size_t)n);
    thread_job *jobs = malloc(sizeof(thread_job) * (size_t)n);
    for (int t = 0; t < n; t++) {
        jobs[t].fn = fn;
        jobs[t].arg = arg;
        jobs[t].t = t;
        if (t > 0 && pthread_create(&th[t], NULL, thread_main, &jobs[t]) != 0) {
            th[t] = 0;
            fn(arg, t); /* could not spawn: run it here */
        }
    }
    fn(arg, 0);
    for (int t = 1; t < n; t++)
        if (th[t]) pthread_join(th[t], NULL);
    free(jobs);
    free(th);
}

/* ---- key transforms, key.rs:135-197 ---- */
static inline uint8_t k_u8(uint8_t v) { return v; }
static inline uint8_t v_u8(uint8_t k) { return k; }
static inline uint16_t k_u16(uint16_t v) { return v; }
static inline uint16_t v_u16(uint16_t k) { return k; }
static inline uint32_t k_u32(uint32_t v) { return v; }
static inline uint32_t v_u32(uint32_t k) { return k; }
static inline uint64_t k_u64(uint64_t v) { return v; }
static inline uint64_t v_u64(uint64_t k) { return k; }
/* signed: XOR the sign bit (key.rs:141-150) */
static inline uint8_t k_i8(int8_t v) { return (uint8_t)((uint8_t)v ^ 0x80u); }
static inline int8_t v_i8(uint8_t k) { return (int8_t)(uint8_t)(k ^ 0x80u); }
static inline uint16_t k_i16(int16_t v) { return (uint16_t)((uint16_t)v ^ 0x8000u); }
static inline int16_t v_i16(uint16_t k) { return (int16_t)(uint16_t)(k ^ 0x8000u); }
static inline uint32_t k_i32(int32_t v) { return (uint32_t)v ^ 0x80000000u; }
static inline int32_t v_i32(uint32_t k) { return (int32_t)(k ^ 0x80000000u); }
static inline uint64_t k_i64(int64_t v) { return (uint64_t)v ^ 0x8000000000000000ull; }
static inline int64_t v_i64(uint64_t k) { return (int64_t)(k ^ 0x8000000000000000ull); }
/* floats: flip the sign bit of positives, every bit of negatives (key.rs:166-197) */
static inline uint32_t k_f32(float v) {
    uint32_t b;
    memcpy(&b, &v, 4);
    return b ^ ((uint32_t)((int32_t)b >> 31) | 0x80000000u);
}
static inline float v_f32(uint32_t k) {
    uint32_t b = k ^ ((uint32_t)~((int32_t)k >> 31) | 0x80000000u);
    float v;
    memcpy(&v, &b, 4);
    return v;
}
static inline uint64_t k_f64(double v) {
    uint64_t b;
    memcpy(&b, &v, 8);
    return b ^ ((uint64_t)((int64_t)b >> 63) | 0x8000000000000000ull);
}
static inline double v_f64(uint64_t k) {
    uint64_t b = k ^ ((uint64_t)~((int64_t)k >> 63) | 0x8000000000000000ull);
    double v;
    memcpy(&v, &b, 8);
    return v;
}

#define T uint8_t
#define U uint8_t
#define SUF u8
#define KEYF k_u8
#define VALF v_u8
#define NBYTES 1
#include "oracle_impl.inc"
#undef T
#undef U
#undef SUF
#undef KEYF
#undef VALF
#undef NBYTES

#define T int8_t
#define U uint8_t
#define SUF i8
#define KEYF k_i8
#define VALF v_i8
#define NBYTES 1
#include "oracle_impl.inc"
#undef T
#undef U
#undef SUF
#undef KEYF
#undef VALF
#undef NBYTES

#define T uint16_t
#define U uint16_t
#define SUF u16
#define KEYF k_u16
#define VALF v_u16
#define NBYTES 2
#include "oracle_impl.inc"
#undef T
#undef U
#undef SUF
#undef KEYF
#undef VALF
#undef NBYTES

#define T int16_t
#define U uint16_t
#define SUF i16
#define KEYF k_i16
#define VALF v_i16
#define NBYTES 2
#include "oracle_impl.inc"
#undef T
#undef U
#undef SUF
#undef KEYF
#undef VALF
#undef NBYTES

#define T uint32_t
#define U uint32_t
#define SUF u32
#define KEYF k_u32
#define VALF v_u32
#define NBYTES 4
#include "oracle_impl.inc"
#undef T
#undef U
#undef SUF
#undef KEYF
#undef VALF
#undef NBYTES

#define T int32_t
#define U uint32_t
#define SUF i32
#define KEYF k_i32
#define VALF v_i32
#define NBYTES 4
#include "oracle_impl.inc"
#undef T
#undef U
#undef SUF
#undef KEYF
#undef VALF
#undef NBYTES

#define T float
#define U uint32_t
#define SUF f32
#define KEYF k_f32
#define VALF v_f32
#define NBYTES 4
#include "oracle_impl.inc"
#undef T
#undef U
#undef SUF
#undef KEYF
#undef VALF
#undef NBYTES

#define T uint64_t
#define U uint64_t
#define SUF u64
#define KEYF k_u64
#define VALF v_u64
#define NBYTES 8
#include "oracle_impl.inc"
#undef T
#undef U
#undef SUF
#undef KEYF
#undef VALF
#undef NBYTES

#define T int64_t
#define U uint64_t
#define SUF i64
#define KEYF k_i64
#define VALF v_i64
#define NBYTES 8
#include "oracle_impl.inc"
#undef T
#undef U
#undef SUF
#undef KEYF
#undef VALF
#undef NBYTES

#define T double
#define U uint64_t
#define SUF f64
#define KEYF k_f64
#define VALF v_f64
#define NBYTES 8
#include "oracle_impl.inc"
#undef T
#undef U
#undef SUF
#undef KEYF
#undef VALF
#undef NBYTES

/* by_key.rs:136-144 and :315-334 — position i gets the element that was at
 * order[i]. Returns 2 on a length mismatch (the crate panics there). */
int tso_apply_order(void *data, size_t n, size_t elem, const uint32_t *order, size_t order_len) {
    if (n != order_len) return 2;
    unsigned char *src = data;
    unsigned char *moved = malloc(n * elem + 1);
    for (size_t i = 0; i < n; i++) memcpy(moved + i * elem, src + (size_t)order[i] * elem, elem);
    memcpy(src, moved, n * elem);
    free(moved);
    return 0;
}

/* histogram.rs:154-158 — passes whose byte varies, as the byte core counts them. */
int tso_counted_passes_u64(const uint64_t *keys, size_t n, int *out) {
    uint64_t vary;
    int some = tso_varying_bits_u64(keys, n, &vary), m = 0;
    for (int p = 0; p < 8; p++)
        if (!some || ((vary >> (8 * p)) & 0xFF) != 0) out[m++] = p;
    return m;
}

/* xorshift64 (13/7/17), the generator of the crate's unit tests
 * (e.g. src/radix/scatter.rs:293-298, src/key.rs:256-262). */
void tso_xorshift64_fill(uint64_t *state, uint64_t *out, size_t n) {
    uint64_t s = *state;
    for (size_t i = 0; i < n; i++) {
        s ^= s << 13;
        s ^= s >> 7;
        s ^= s << 17;
        out[i] = s;
    }
    *state = s;
}
