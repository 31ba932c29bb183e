// ts_staging.h — host threads that copy between a caller's pageable memory
// and the context's pinned staging slots.
//
// A copy from pageable host memory cannot be a DMA of its own: the CUDA driver
// copies it through its own pinned buffer on the calling thread, at about a
// quarter of what PCIe carries. The host-slice pipeline instead copies each
// piece into one of its pinned slots with several threads at once, and the
// DMA of that slot overlaps the threads' copy of the next piece.
#pragma once

#include <algorithm>
#include <condition_variable>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

namespace ts {

class CopyPool {
  public:
    explicit CopyPool(int workers) {
        for (int w = 0; w < workers; ++w) threads_.emplace_back([this, w] { run(w); });
    }
    ~CopyPool() {
        {
            std::lock_guard<std::mutex> g(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& t : threads_) t.join();
    }
    CopyPool(const CopyPool&) = delete;
    CopyPool& operator=(const CopyPool&) = delete;

    // dst[0, bytes) = src[0, bytes), split over the workers and the caller;
    // returns when every part is done
    void copy(void* dst, const void* src, size_t bytes) {
        const int parts = (int)threads_.size() + 1;
        if (bytes < ((size_t)1 << 20) || parts == 1) {
            std::memcpy(dst, src, bytes);
            return;
        }
        {
            std::lock_guard<std::mutex> g(mu_);
            dst_ = (char*)dst;
            src_ = (const char*)src;
            bytes_ = bytes;
            pending_ = (int)threads_.size();
            ++gen_;
        }
        cv_.notify_all();
        part(parts - 1, parts);
        std::unique_lock<std::mutex> l(mu_);
        done_.wait(l, [this] { return pending_ == 0; });
    }

  private:
    void part(int w, int parts) {
        const size_t b = bytes_ * (size_t)w / parts / 64 * 64;
        const size_t e = w + 1 == parts ? bytes_ : bytes_ * (size_t)(w + 1) / parts / 64 * 64;
        if (e > b) std::memcpy(dst_ + b, src_ + b, e - b);
    }
    void run(int w) {
        unsigned seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> l(mu_);
                cv_.wait(l, [&] { return stop_ || gen_ != seen; });
                if (stop_) return;
                seen = gen_;
            }
            part(w, (int)threads_.size() + 1);
            {
                std::lock_guard<std::mutex> g(mu_);
                if (--pending_ == 0) done_.notify_one();
            }
        }
    }

    std::vector<std::thread> threads_;
    std::mutex mu_;
    std::condition_variable cv_, done_;
    char* dst_ = nullptr;
    const char* src_ = nullptr;
    size_t bytes_ = 0;
    unsigned gen_ = 0;
    int pending_ = 0;
    bool stop_ = false;
};

// worker threads for a context's pool: the caller copies a part as well
inline int copy_pool_workers() {
    const unsigned hc = std::thread::hardware_concurrency();
    return (int)std::min(7u, std::max(1u, hc / 2) - 1u);
}

}  // namespace ts
