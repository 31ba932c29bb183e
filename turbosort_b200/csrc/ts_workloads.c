/*
 * ts_workloads.c — seeded synthetic inputs for the benchmark configurations.
 *
 * xorshift64 (shifts 13/7/17), the generator of the turbosort crate's own
 * tests (src/radix/scatter.rs:293-298, src/key.rs:256-262); a 32-bit key is
 * the low half of one output (src/radix/scatter.rs:308).
 */
#include <stddef.h>
#include <stdint.h>
#include <string.h>

static inline uint64_t xs_next(uint64_t *s) {
    uint64_t x = *s;
    x ^= x << 13;
    x ^= x >> 7;
    x ^= x << 17;
    *s = x;
    return x;
}

void tsw_xorshift64(uint64_t *state, uint64_t *out, size_t n) {
    uint64_t s = *state;
    for (size_t i = 0; i < n; i++) out[i] = xs_next(&s);
    *state = s;
}

/* dist 0: full-entropy words; 1: AND of three words (low entropy);
 * 2: confined to 16 bits in the low end. */
void tsw_gen_u32(uint64_t seed, int dist, uint32_t *out, size_t n) {
    uint64_t s = seed ? seed : 1;
    for (size_t i = 0; i < n; i++) {
        uint64_t r = xs_next(&s);
        if (dist == 1) r &= xs_next(&s) & xs_next(&s);
        if (dist == 2) r &= 0xFFFF;
        out[i] = (uint32_t)r;
    }
}

void tsw_gen_u64(uint64_t seed, int dist, uint64_t *out, size_t n) {
    uint64_t s = seed ? seed : 1;
    for (size_t i = 0; i < n; i++) {
        uint64_t r = xs_next(&s);
        if (dist == 1) r &= xs_next(&s) & xs_next(&s);
        if (dist == 2) r &= 0xFFFF;
        out[i] = r;
    }
}

/* f32 bit patterns of distribution `dist`, with specials mixed in by a class
 * draw per element: 1% NaN (either sign, random non-zero payload), 1% +-0.0,
 * 0.5% +-inf, the rest the distribution's bit pattern. */
void tsw_gen_f32_bits(uint64_t seed, int dist, uint32_t *out, size_t n) {
    uint64_t s = seed ? seed : 1;
    for (size_t i = 0; i < n; i++) {
        uint64_t r = xs_next(&s);
        if (dist == 1) r &= xs_next(&s) & xs_next(&s);
        if (dist == 2) r &= 0xFFFF;
        uint64_t c = xs_next(&s);
        uint32_t cls = (uint32_t)((c >> 32) % 2000u); /* units of 0.05% */
        uint32_t sign = (uint32_t)(c & 1u) << 31;
        uint32_t bits = (uint32_t)r;
        if (cls < 20) { /* NaN */
            uint32_t payload = (uint32_t)(c >> 1) & 0x7FFFFFu;
            bits = sign | 0x7F800000u | (payload ? payload : 1u);
        } else if (cls < 40) { /* +-0.0 */
            bits = sign;
        } else if (cls < 50) { /* +-inf */
            bits = sign | 0x7F800000u;
        }
        out[i] = bits;
    }
}
