/* The CPU oracle (oracle/turbosort_oracle.c) under AddressSanitizer and
 * UndefinedBehaviorSanitizer: every key type at the crate's tier-boundary
 * sizes and shapes through sort, sort_parallel, sort_by_key and
 * apply_order, each result checked here (sorted radix keys, the same
 * multiset, order() a stable permutation, sort_parallel == sort). */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

int tso_apply_order(void *data, size_t n, size_t elem, const uint32_t *order, size_t order_len);

static uint64_t rng_state = 0x9E3779B97F4A7C15ull;
static uint64_t rnd(void) {
    rng_state ^= rng_state << 13;
    rng_state ^= rng_state >> 7;
    rng_state ^= rng_state << 17;
    return rng_state;
}

static const size_t SIZES[] = {0, 1, 2, 15, 16, 17, 47, 48, 63, 64, 65, 511, 512, 513, 4095, 4096, 4097, 65537, 300001};
enum { RANDOM, FEW, ASC, DESC, CONST, TOP_ONLY, NSHAPES };

#define DEFINE_CHECK(T, SUF, U)                                                                             \
    void tso_sort_##SUF(T *data, size_t n);                                                                 \
    void tso_sort_parallel_##SUF(T *data, size_t n, int threads);                                           \
    int tso_sort_by_key_##SUF(const T *keys, size_t n, uint32_t *order);                                    \
    void tso_radix_keys_##SUF(const T *in, U *out, size_t n);                                               \
    static int check_##SUF(void) {                                                                          \
        for (size_t si = 0; si < sizeof SIZES / sizeof SIZES[0]; ++si) {                                    \
            const size_t n = SIZES[si];                                                                     \
            U *bits = malloc(n * sizeof(U) + 8), *rk = malloc(n * sizeof(U) + 8);                           \
            T *a = malloc(n * sizeof(T) + 8), *b = malloc(n * sizeof(T) + 8), *orig = malloc(n * sizeof(T) + 8); \
            uint32_t *order = malloc(n * 4 + 8);                                                            \
            unsigned char *seen = malloc(n + 1);                                                            \
            for (int shape = 0; shape < NSHAPES; ++shape) {                                                 \
                for (size_t i = 0; i < n; ++i) {                                                            \
                    U v = (U)rnd();                                                                         \
                    if (shape == FEW) v = (U)(v % 5u);                                                      \
                    if (shape == CONST) v = (U)12345u;                                                      \
                    if (shape == TOP_ONLY) v = (U)((U)(v & 0xFFu) << (8 * sizeof(U) - 8));                  \
                    bits[i] = v;                                                                            \
                }                                                                                           \
                memcpy(a, bits, n * sizeof(T));                                                             \
                if (shape == ASC || shape == DESC) {                                                        \
                    tso_sort_##SUF(a, n);                                                                   \
                    if (shape == DESC)                                                                      \
                        for (size_t i = 0; i < n / 2; ++i) {                                                \
                            T t = a[i];                                                                     \
                            a[i] = a[n - 1 - i];                                                            \
                            a[n - 1 - i] = t;                                                               \
                        }                                                                                   \
                }                                                                                           \
                memcpy(orig, a, n * sizeof(T));                                                             \
                memcpy(b, a, n * sizeof(T));                                                                \
                U sum0 = 0, xor0 = 0, sum1 = 0, xor1 = 0;                                                   \
                memcpy(bits, a, n * sizeof(T));                                                             \
                for (size_t i = 0; i < n; ++i) sum0 += bits[i], xor0 ^= bits[i];                            \
                tso_sort_##SUF(a, n);                                                                       \
                memcpy(bits, a, n * sizeof(T));                                                             \
                for (size_t i = 0; i < n; ++i) sum1 += bits[i], xor1 ^= bits[i];                            \
                if (sum0 != sum1 || xor0 != xor1) return printf(#SUF " n=%zu shape=%d: not a permutation\n", n, shape), 1; \
                tso_radix_keys_##SUF(a, rk, n);                                                             \
                for (size_t i = 1; i < n; ++i)                                                              \
                    if (rk[i - 1] > rk[i]) return printf(#SUF " n=%zu shape=%d: unsorted at %zu\n", n, shape, i), 1; \
                tso_sort_parallel_##SUF(b, n, 4);                                                           \
                if (memcmp(a, b, n * sizeof(T)) != 0) return printf(#SUF " n=%zu shape=%d: parallel differs\n", n, shape), 1; \
                if (n <= 0xffffffffu) {                                                                     \
                    if (tso_sort_by_key_##SUF(orig, n, order) != 0) return printf(#SUF " by_key failed\n"), 1; \
                    memset(seen, 0, n + 1);                                                                 \
                    tso_radix_keys_##SUF(orig, rk, n);                                                      \
                    for (size_t i = 0; i < n; ++i) {                                                        \
                        if (order[i] >= n || seen[order[i]]) return printf(#SUF " order not a permutation\n"), 1; \
                        seen[order[i]] = 1;                                                                 \
                        if (i > 0) {                                                                        \
                            const U p = rk[order[i - 1]], q = rk[order[i]];                                 \
                            if (p > q || (p == q && order[i - 1] > order[i]))                               \
                                return printf(#SUF " n=%zu shape=%d: order unstable at %zu\n", n, shape, i), 1; \
                        }                                                                                   \
                    }                                                                                       \
                    memcpy(b, orig, n * sizeof(T));                                                         \
                    if (tso_apply_order(b, n, sizeof(T), order, n) != 0) return printf("apply_order failed\n"), 1; \
                    if (memcmp(a, b, n * sizeof(T)) != 0) return printf(#SUF " apply_order(order) != sort\n"), 1; \
                }                                                                                           \
            }                                                                                               \
            free(bits), free(rk), free(a), free(b), free(orig), free(order), free(seen);                    \
        }                                                                                                   \
        return 0;                                                                                           \
    }

DEFINE_CHECK(uint8_t, u8, uint8_t)
DEFINE_CHECK(int8_t, i8, uint8_t)
DEFINE_CHECK(uint16_t, u16, uint16_t)
DEFINE_CHECK(int16_t, i16, uint16_t)
DEFINE_CHECK(uint32_t, u32, uint32_t)
DEFINE_CHECK(int32_t, i32, uint32_t)
DEFINE_CHECK(float, f32, uint32_t)
DEFINE_CHECK(uint64_t, u64, uint64_t)
DEFINE_CHECK(int64_t, i64, uint64_t)
DEFINE_CHECK(double, f64, uint64_t)

int main(void) {
    if (check_u8() || check_i8() || check_u16() || check_i16() || check_u32() || check_i32() || check_f32() ||
        check_u64() || check_i64() || check_f64())
        return 1;
    printf("ok\n");
    return 0;
}
