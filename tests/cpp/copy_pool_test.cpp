// The host copy pool of the transfer pipeline (turbosort_b200/csrc/ts_staging.h):
// every byte of every copy lands, for sizes around its split and threshold
// points, with 0 to 7 worker threads and many copies in a row.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "ts_staging.h"

int main() {
    const size_t sizes[] = {0, 1, 63, 64, 65, (1u << 20) - 1, 1u << 20, (1u << 20) + 1, (33u << 20) + 7};
    std::vector<uint8_t> src((33u << 20) + 64), dst(src.size());
    uint64_t x = 0x9E3779B97F4A7C15ull;
    for (auto& b : src) {
        x ^= x << 13;
        x ^= x >> 7;
        x ^= x << 17;
        b = (uint8_t)x;
    }
    for (int workers : {0, 1, 3, 7}) {
        ts::CopyPool pool(workers);
        for (int round = 0; round < 3; ++round)
            for (size_t n : sizes)
                for (size_t off : {(size_t)0, (size_t)3}) {
                    std::memset(dst.data(), 0xA5, dst.size());
                    pool.copy(dst.data() + off, src.data() + round, n);
                    if (std::memcmp(dst.data() + off, src.data() + round, n) != 0) {
                        std::printf("mismatch: workers %d size %zu offset %zu\n", workers, n, off);
                        return 1;
                    }
                    for (size_t i = 0; i < off; ++i)
                        if (dst[i] != 0xA5) return 2;
                    if (dst[off + n] != 0xA5) {
                        std::printf("wrote past the end: workers %d size %zu\n", workers, n);
                        return 3;
                    }
                }
        for (int k = 0; k < 2000; ++k) pool.copy(dst.data(), src.data(), (1u << 20) + (size_t)k);
        if (std::memcmp(dst.data(), src.data(), (1u << 20) + 1999) != 0) return 4;
    }
    std::printf("ok\n");
    return 0;
}
