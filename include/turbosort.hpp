// turbosort.hpp — the turbosort crate's public API in C++, over the C ABI of
// libturbosort_b200.so (turbosort.h). Header-only.
//
//   turbosort::sort(data, n)                       src/lib.rs:99
//   turbosort::sort_with_buffer(data, n, buf, m)   src/lib.rs:122  throws std::length_error
//                                                  "buffer too small: need N, got M"
//   turbosort::sort_parallel(data, n)              src/lib.rs:224
//   turbosort::sort_by_key(data, n, key)           src/lib.rs:152  stable
//   turbosort::sort_by_key_with_buffer(data, n, buffer, key)   src/lib.rs:196
//   turbosort::SortByKeyBuffer<T, K>::order() / apply_order() / capacity()
//                                                  src/by_key.rs:51-145
//
// The sortable key types are the crate's ten (src/key.rs:64-77). Floats sort
// in total_cmp order, every bit pattern preserved. Slices are host memory;
// each call copies to the GPU, sorts there and copies back. Calls from one
// thread share a per-thread context (a CUDA stream and device scratch that
// grows to the largest sort). Errors of the C ABI are thrown as
// turbosort::Error; the crate's two panics keep their messages.
#pragma once

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <algorithm>
#include <numeric>
#include <vector>

#include "turbosort.h"

namespace turbosort {

class Error : public std::runtime_error {
   public:
    Error(ts_status s, const std::string& what) : std::runtime_error(what), status(s) {}
    ts_status status;
};

namespace detail {

// One context per host thread, on device 0 (a context is not thread-safe).
class Context {
   public:
    Context() {
        ts_status s = ts_ctx_create(0, &ctx_);
        if (s != TS_OK) throw Error(s, std::string("turbosort: ") + ts_status_str(s));
    }
    ~Context() { ts_ctx_destroy(ctx_); }
    Context(const Context&) = delete;
    Context& operator=(const Context&) = delete;
    ts_ctx* get() const { return ctx_; }

   private:
    ts_ctx* ctx_ = nullptr;
};

inline ts_ctx* thread_ctx() {
    thread_local Context ctx;
    return ctx.get();
}

inline void check(ts_ctx* c, ts_status s) {
    if (s == TS_OK) return;
    std::string msg = ts_ctx_last_error(c);
    if (msg.empty()) msg = ts_status_str(s);
    if (s == TS_ERR_BUFFER_TOO_SMALL) throw std::length_error(msg);
    if (s == TS_ERR_LENGTH_MISMATCH) throw std::invalid_argument(msg);
    throw Error(s, msg);
}

template <class T>
struct Key;  // the C entry points of each sortable type

#define TURBOSORT_KEY(T, SUF)                                                                             \
    template <>                                                                                           \
    struct Key<T> {                                                                                       \
        static ts_status sort(ts_ctx* c, T* d, size_t n) { return ts_sort_##SUF(c, d, n); }              \
        static ts_status sort_with_buffer(ts_ctx* c, T* d, size_t n, T* b, size_t m) {                    \
            return ts_sort_with_buffer_##SUF(c, d, n, b, m);                                             \
        }                                                                                                 \
        static ts_status sort_parallel(ts_ctx* c, T* d, size_t n) { return ts_sort_parallel_##SUF(c, d, n); } \
        static ts_status order(ts_ctx* c, const T* k, size_t n, uint32_t* o) {                          \
            return ts_sort_keys_order_##SUF(c, k, n, o);                                                 \
        }                                                                                                 \
    };
TURBOSORT_KEY(uint8_t, u8)
TURBOSORT_KEY(uint16_t, u16)
TURBOSORT_KEY(uint32_t, u32)
TURBOSORT_KEY(uint64_t, u64)
TURBOSORT_KEY(int8_t, i8)
TURBOSORT_KEY(int16_t, i16)
TURBOSORT_KEY(int32_t, i32)
TURBOSORT_KEY(int64_t, i64)
TURBOSORT_KEY(float, f32)
TURBOSORT_KEY(double, f64)
#undef TURBOSORT_KEY

// to_radix_key (src/key.rs:135-197), for the host-side fallback above u32::MAX.
template <class K>
inline auto radix_key(K k) {
    if constexpr (std::is_same_v<K, float>) {
        uint32_t b;
        static_assert(sizeof b == sizeof k);
        __builtin_memcpy(&b, &k, 4);
        return b ^ ((uint32_t)((int32_t)b >> 31) | 0x80000000u);
    } else if constexpr (std::is_same_v<K, double>) {
        uint64_t b;
        __builtin_memcpy(&b, &k, 8);
        return b ^ ((uint64_t)((int64_t)b >> 63) | 0x8000000000000000ull);
    } else if constexpr (std::is_signed_v<K>) {
        using U = std::make_unsigned_t<K>;
        return (U)((U)k ^ ((U)1 << (8 * sizeof(U) - 1)));
    } else {
        return k;
    }
}

}  // namespace detail

/// Sort `data[0..n)` ascending (src/lib.rs:99).
template <class T>
void sort(T* data, size_t n) {
    ts_ctx* c = detail::thread_ctx();
    detail::check(c, detail::Key<T>::sort(c, data, n));
}
template <class T>
void sort(std::vector<T>& v) {
    sort(v.data(), v.size());
}

/// Sort with a caller's buffer of at least n elements (src/lib.rs:122).
template <class T>
void sort_with_buffer(T* data, size_t n, T* buf, size_t buf_len) {
    ts_ctx* c = detail::thread_ctx();
    detail::check(c, detail::Key<T>::sort_with_buffer(c, data, n, buf, buf_len));
}
template <class T>
void sort_with_buffer(std::vector<T>& v, std::vector<T>& buf) {
    sort_with_buffer(v.data(), v.size(), buf.data(), buf.size());
}

/// The crate's multi-core sort (src/lib.rs:224): the same device sort.
template <class T>
void sort_parallel(T* data, size_t n) {
    ts_ctx* c = detail::thread_ctx();
    detail::check(c, detail::Key<T>::sort_parallel(c, data, n));
}
template <class T>
void sort_parallel(std::vector<T>& v) {
    sort_parallel(v.data(), v.size());
}

/// Reusable memory for sort_by_key_with_buffer (src/by_key.rs:51-145): the
/// keys, the order of the last sort, and a context whose device scratch grows
/// to the longest slice sorted through it.
template <class T, class K>
class SortByKeyBuffer {
   public:
    SortByKeyBuffer() {
        ts_status s = ts_ctx_create(0, &ctx_);
        if (s != TS_OK) throw Error(s, std::string("turbosort: ") + ts_status_str(s));
    }
    explicit SortByKeyBuffer(size_t capacity) : SortByKeyBuffer() {
        keys_.reserve(capacity);
        order_.reserve(capacity);
        detail::check(ctx_, ts_ctx_reserve(ctx_, capacity, sizeof(K), 1));
    }
    ~SortByKeyBuffer() { ts_ctx_destroy(ctx_); }
    SortByKeyBuffer(const SortByKeyBuffer&) = delete;
    SortByKeyBuffer& operator=(const SortByKeyBuffer&) = delete;

    /// Elements it can sort without growing (src/by_key.rs:84-90).
    size_t capacity() const {
        return std::min({keys_.capacity(), order_.capacity(), ts_ctx_capacity(ctx_, sizeof(K), 1)});
    }

    /// Position i of the last sorted slice holds the element that was at
    /// order()[i]; empty before the first sort and after a slice of more than
    /// u32::MAX elements (src/by_key.rs:92-110).
    const std::vector<uint32_t>& order() const { return order_; }

    /// Put `other[0..n)` in the order of the last sort (src/by_key.rs:136-144).
    /// Trivially copyable elements are gathered on the device; others are
    /// moved on the host through `scratch`, which is left empty.
    template <class U>
    void apply_order(U* other, size_t n, std::vector<U>& scratch) const {
        if (n != order_.size())
            throw std::invalid_argument("apply_order: the slice's length differs from the last sorted slice's");
        scratch.clear();
        if (n == 0) return;
        if constexpr (std::is_trivially_copyable_v<U>) {
            detail::check(ctx_, ts_apply_order(ctx_, other, n, sizeof(U), order_.data(), n));
        } else {
            scratch.reserve(n);
            for (size_t i = 0; i < n; ++i) scratch.push_back(std::move(other[order_[i]]));
            for (size_t i = 0; i < n; ++i) other[i] = std::move(scratch[i]);
            scratch.clear();
        }
    }
    template <class U>
    void apply_order(std::vector<U>& other, std::vector<U>& scratch) const {
        apply_order(other.data(), other.size(), scratch);
    }

   private:
    template <class T2, class K2, class F>
    friend void sort_by_key_with_buffer(T2* data, size_t n, SortByKeyBuffer<T2, K2>& buffer, F key);

    ts_ctx* ctx_ = nullptr;
    std::vector<K> keys_;
    std::vector<uint32_t> order_;
    std::vector<T> moved_;
};

/// Stable sort of data[0..n) by key(x), called once per element, with memory
/// kept in `buffer` (src/lib.rs:196, src/by_key.rs:175-235).
template <class T, class K, class F>
void sort_by_key_with_buffer(T* data, size_t n, SortByKeyBuffer<T, K>& buffer, F key) {
    buffer.keys_.clear();
    buffer.keys_.reserve(n);
    for (size_t i = 0; i < n; ++i) buffer.keys_.push_back(static_cast<K>(key(data[i])));
    if (n < 2) {
        buffer.order_.assign(n, 0u);
        std::iota(buffer.order_.begin(), buffer.order_.end(), 0u);
        return;
    }
    if (n > 0xffffffffull) {  // order() stays empty; the host's stable sort instead
        buffer.order_.clear();
        std::vector<size_t> idx(n);
        std::iota(idx.begin(), idx.end(), size_t{0});
        std::stable_sort(idx.begin(), idx.end(), [&](size_t a, size_t b) {
            return detail::radix_key(buffer.keys_[a]) < detail::radix_key(buffer.keys_[b]);
        });
        buffer.moved_.clear();
        for (size_t i : idx) buffer.moved_.push_back(std::move(data[i]));
        std::move(buffer.moved_.begin(), buffer.moved_.end(), data);
        buffer.moved_.clear();
        return;
    }
    buffer.order_.resize(n);
    detail::check(buffer.ctx_, detail::Key<K>::order(buffer.ctx_, buffer.keys_.data(), n, buffer.order_.data()));
    buffer.apply_order(data, n, buffer.moved_);
}
template <class T, class K, class F>
void sort_by_key_with_buffer(std::vector<T>& v, SortByKeyBuffer<T, K>& buffer, F key) {
    sort_by_key_with_buffer(v.data(), v.size(), buffer, key);
}

/// Stable sort by key with a fresh buffer (src/lib.rs:152).
template <class T, class F>
void sort_by_key(T* data, size_t n, F key) {
    using K = std::decay_t<decltype(key(std::declval<const T&>()))>;
    SortByKeyBuffer<T, K> buffer;
    sort_by_key_with_buffer(data, n, buffer, key);
}
template <class T, class F>
void sort_by_key(std::vector<T>& v, F key) {
    sort_by_key(v.data(), v.size(), key);
}

}  // namespace turbosort
