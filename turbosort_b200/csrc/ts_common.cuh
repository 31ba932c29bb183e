// ts_common.cuh — key traits, device helpers and the plan shared by every
// kernel of the B200 radix sort.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace ts {

// ---------------------------------------------------------------------------
// Order-preserving key transform of the crate (src/key.rs:135-197), on the
// value's bits. XF 0: unsigned (identity); 1: signed (XOR the sign bit);
// 2: IEEE float (flip the sign bit of positives, every bit of negatives).
// Integer operations only, so NaN payloads and -0.0 pass through untouched.
// ---------------------------------------------------------------------------
template <typename U>
struct Bits;
template <> struct Bits<uint8_t>  { using S = int8_t;  static constexpr int W = 8;  };
template <> struct Bits<uint16_t> { using S = int16_t; static constexpr int W = 16; };
template <> struct Bits<uint32_t> { using S = int32_t; static constexpr int W = 32; };
template <> struct Bits<uint64_t> { using S = int64_t; static constexpr int W = 64; };

template <typename U, int XF>
__host__ __device__ __forceinline__ U to_key(U b) {
    constexpr U SIGN = (U)((U)1 << (Bits<U>::W - 1));
    if constexpr (XF == 0) {
        return b;
    } else if constexpr (XF == 1) {
        return (U)(b ^ SIGN);
    } else {
        U m = (U)((typename Bits<U>::S)b >> (Bits<U>::W - 1));
        return (U)(b ^ (U)(m | SIGN));
    }
}

template <typename U, int XF>
__host__ __device__ __forceinline__ U from_key(U k) {
    constexpr U SIGN = (U)((U)1 << (Bits<U>::W - 1));
    if constexpr (XF == 0) {
        return k;
    } else if constexpr (XF == 1) {
        return (U)(k ^ SIGN);
    } else {
        U m = (U)~(U)((typename Bits<U>::S)k >> (Bits<U>::W - 1));
        return (U)(k ^ (U)(m | SIGN));
    }
}

template <typename U>
__host__ __device__ __forceinline__ uint32_t digit_of(U k, int shift, uint32_t mask) {
    return (uint32_t)(k >> shift) & mask;
}

// ---------------------------------------------------------------------------
// Limits and status.
// ---------------------------------------------------------------------------
constexpr int MAX_PASSES = 16;         // 64-bit keys at 4-bit digits
constexpr uint32_t LB_FLAG_AGG = 1u << 30;   // look-back: tile count only
constexpr uint32_t LB_FLAG_INC = 2u << 30;   // look-back: inclusive prefix
constexpr uint32_t LB_VALUE = (1u << 30) - 1;
constexpr uint32_t SPIN_LIMIT = 1u << 20;    // bounded waits (about a second), then TS_ERR_TIMEOUT
constexpr int LB_WINDOW = 4;                 // look-back entries loaded per round trip (4 beat 8, 16, 32 on a B200)
constexpr uint32_t ERR_TIMEOUT = 1u;
constexpr uint32_t ERR_BOUNDS = 2u;

// What the upfront scan found (written by k_scan, read by k_hist).
struct ScanState {
    unsigned long long diff;    // OR of (key ^ first key): the bits that vary
    unsigned int flags;         // bit 0: some pair descends; bit 1: some pair ascends
    unsigned int hist_done;     // k_hist CTAs that have added their counts
};
constexpr unsigned SCAN_NOT_ASC = 1u;
constexpr unsigned SCAN_NOT_DESC = 2u;

enum PlanMode : int { MODE_SORT = 0, MODE_SORTED = 1, MODE_REVERSE = 2 };

// The device-side plan: which digit passes run, decided on the GPU from the
// upfront histograms so that no host round trip sits between the kernels.
struct Plan {
    int mode;
    int n_live;                  // live digit passes, least significant first
    int pass[MAX_PASSES];        // digit index of the j-th live pass
    int divert_shift;            // > 0: only digits from this bit up were sorted; runs left to finish
    int pad;
};

// ---------------------------------------------------------------------------
// PTX helpers: relaxed GPU-scope accesses for the look-back words (they
// bypass the non-coherent L1), and the bulk-copy / mbarrier primitives.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t ld_relaxed_gpu(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed_gpu(uint32_t* p, uint32_t v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_volatile_u64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ uint32_t ld_volatile_u32(const unsigned int* p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}
// One bulk global->shared copy (no multicast), completing on `bar`.
// Both addresses 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst_smem, const void* src_gmem, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst_smem)),
        "l"(src_gmem), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}
// Starts an asynchronous copy of global bytes [begin, end) into L2, narrowed
// to 16-byte bounds (the bulk prefetch's rule), so it never touches a byte
// outside the range.
__device__ __forceinline__ void prefetch_l2(const void* begin, const void* end) {
    const uintptr_t a = ((uintptr_t)begin + 15) & ~(uintptr_t)15;
    const uintptr_t e = (uintptr_t)end & ~(uintptr_t)15;
    if (e > a)
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"((uint32_t)(e - a)) : "memory");
}

// Bounded wait on an mbarrier phase; returns false if the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase) {
    uint32_t ok = 0;
    for (uint32_t i = 0; i < SPIN_LIMIT; ++i) {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(smem_addr(bar)), "r"(phase)
            : "memory");
        if (ok) return true;
    }
    return false;
}

// Programmatic dependent launch: a kernel launched with programmatic stream
// serialization may start before its predecessor in the stream has finished;
// dep_wait() blocks until that predecessor has completed and its writes are
// visible (a no-op for an ordinary launch), and dep_release() lets the next
// such kernel start launching early. Every kernel of the LSD chain calls
// dep_wait() before it touches memory.
__device__ __forceinline__ void dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void dep_release() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

}  // namespace ts
