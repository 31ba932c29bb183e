// CUB's device radix sort (the CUDA toolkit's library sort) timed on the same
// keys as bench.py's headline workload: 2^lg uniformly random u32 keys from
// the xorshift64 generator seeded 0x9E3779B97F4A7C15, keys only, device
// resident, CUDA events around each sort, 3 warm-up sorts. A reference point
// for the onesweep kernel, not part of the library.
//   nvcc -gencode arch=compute_100a,code=sm_100a -O3 -std=c++17 \
//        baseline/cub_radix_sort.cu -o baseline/_ref/cub_radix_sort
//   baseline/_ref/cub_radix_sort 28
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

int main(int argc, char** argv) {
    const int lg = argc > 1 ? atoi(argv[1]) : 28;
    const size_t n = (size_t)1 << lg;
    std::vector<uint32_t> h(n);
    uint64_t x = 0x9E3779B97F4A7C15ull;
    for (size_t i = 0; i < n; ++i) {
        x ^= x << 13;
        x ^= x >> 7;
        x ^= x << 17;
        h[i] = (uint32_t)x;
    }
    uint32_t *a, *b, *m;
    if (cudaMalloc(&a, n * 4) != cudaSuccess || cudaMalloc(&b, n * 4) != cudaSuccess ||
        cudaMalloc(&m, n * 4) != cudaSuccess) {
        printf("cudaMalloc failed\n");
        return 1;
    }
    cudaMemcpy(m, h.data(), n * 4, cudaMemcpyHostToDevice);
    size_t temp_bytes = 0;
    void* temp = nullptr;
    cub::DoubleBuffer<uint32_t> db(a, b);
    cub::DeviceRadixSort::SortKeys(temp, temp_bytes, db, (int)n);
    cudaMalloc(&temp, temp_bytes);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int warm = 3, reps = 10;
    float total = 0.f, best = 1e30f;
    cub::DoubleBuffer<uint32_t> last(a, b);
    for (int r = 0; r < warm + reps; ++r) {
        cudaMemcpy(a, m, n * 4, cudaMemcpyDeviceToDevice);
        cub::DoubleBuffer<uint32_t> d(a, b);
        cudaEventRecord(e0);
        cub::DeviceRadixSort::SortKeys(temp, temp_bytes, d, (int)n);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (r >= warm) {
            total += ms;
            best = std::min(best, ms);
        }
        last = d;
    }
    std::vector<uint32_t> o(n);
    cudaMemcpy(o.data(), last.Current(), n * 4, cudaMemcpyDeviceToHost);
    std::sort(h.begin(), h.end());
    printf("cub::DeviceRadixSort::SortKeys u32 2^%d: mean %.3f ms, best %.3f ms, %.1f GKeys/s, sorted=%d, %s\n", lg,
           total / reps, best, n / (total / reps) / 1e6, (int)(o == h), cudaGetErrorString(cudaGetLastError()));
    return 0;
}
