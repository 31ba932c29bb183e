// The crate's README and doc examples through the C++ API (turbosort.hpp),
// plus larger slices checked against the standard library. Exits non-zero on
// the first mismatch.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <random>
#include <string>
#include <utility>
#include <vector>

#include "turbosort.hpp"

#define CHECK(cond)                                                        \
    do {                                                                   \
        if (!(cond)) {                                                     \
            std::fprintf(stderr, "FAILED %s:%d: %s\n", __FILE__, __LINE__, #cond); \
            return 1;                                                      \
        }                                                                  \
    } while (0)

static uint32_t bits(float f) {
    uint32_t b;
    std::memcpy(&b, &f, 4);
    return b;
}

int main() {
    // src/lib.rs:18-20
    std::vector<uint32_t> v{5, 3, 8, 1, 9, 2, 7, 4, 6};
    turbosort::sort(v);
    CHECK((v == std::vector<uint32_t>{1, 2, 3, 4, 5, 6, 7, 8, 9}));
    // src/lib.rs:82-84
    std::vector<int32_t> s{3, -1, 4, -1, 5, -9};
    turbosort::sort(s);
    CHECK((s == std::vector<int32_t>{-9, -1, -1, 3, 4, 5}));
    // src/lib.rs:92-96: -inf, -0.0, +0.0, 1.0, NaN
    std::vector<float> f{1.0f, std::numeric_limits<float>::quiet_NaN(), -0.0f, 0.0f,
                         -std::numeric_limits<float>::infinity()};
    turbosort::sort(f);
    CHECK(std::isinf(f[0]) && f[0] < 0);
    CHECK(bits(f[1]) == 0x80000000u && bits(f[2]) == 0u && f[3] == 1.0f && std::isnan(f[4]));
    // src/lib.rs:116-119 and the buffer panic (src/dispatch.rs:78-83)
    std::vector<uint64_t> d{42, 7, 99, 1, 0}, buf(5);
    turbosort::sort_with_buffer(d, buf);
    CHECK((d == std::vector<uint64_t>{0, 1, 7, 42, 99}));
    std::vector<uint64_t> small(4);
    bool threw = false;
    try {
        turbosort::sort_with_buffer(d, small);
    } catch (const std::length_error& e) {
        threw = std::string(e.what()) == "buffer too small: need 5, got 4";
    }
    CHECK(threw);
    // README.md:53-60: stable sort by key, then through a reused buffer
    std::vector<std::pair<std::string, uint32_t>> people{{"bob", 31}, {"alice", 25}, {"carol", 31}, {"dave", 25}};
    turbosort::sort_by_key(people, [](const auto& p) { return p.second; });
    CHECK(people[0].first == "alice" && people[1].first == "dave" && people[2].first == "bob" &&
          people[3].first == "carol");
    turbosort::SortByKeyBuffer<std::pair<std::string, uint32_t>, uint32_t> buffer;
    turbosort::sort_by_key_with_buffer(people, buffer, [](const auto& p) { return (uint32_t)p.first.size(); });
    CHECK(people[0].first == "bob" && people[1].first == "dave" && people[2].first == "alice" &&
          people[3].first == "carol");
    // README.md:61-67: order() and apply_order on a parallel slice
    std::vector<uint32_t> ids{30, 10, 20};
    std::vector<std::string> names{"c", "a", "b"}, scratch;
    turbosort::SortByKeyBuffer<uint32_t, uint32_t> id_buffer;
    turbosort::sort_by_key_with_buffer(ids, id_buffer, [](uint32_t id) { return id; });
    CHECK((id_buffer.order() == std::vector<uint32_t>{1, 2, 0}));
    id_buffer.apply_order(names, scratch);
    CHECK(names[0] == "a" && names[1] == "b" && names[2] == "c" && scratch.empty());
    std::vector<std::string> wrong{"x", "y"};
    threw = false;
    try {
        id_buffer.apply_order(wrong, scratch);
    } catch (const std::invalid_argument& e) {
        threw = std::string(e.what()) == "apply_order: the slice's length differs from the last sorted slice's";
    }
    CHECK(threw);
    // a large slice against std::sort
    std::mt19937_64 rng(7);
    std::vector<uint32_t> big(1 << 20);
    for (auto& x : big) x = (uint32_t)rng();
    std::vector<uint32_t> want = big;
    std::sort(want.begin(), want.end());
    turbosort::sort_parallel(big);
    CHECK(big == want);
    // records by a few-valued u64 key against std::stable_sort
    struct Rec {
        uint64_t id;
        uint32_t a, b;
    };
    std::vector<Rec> recs(300000);
    for (size_t i = 0; i < recs.size(); ++i) recs[i] = Rec{i, (uint32_t)rng(), (uint32_t)(rng() % 50)};
    std::vector<Rec> ref = recs;
    std::stable_sort(ref.begin(), ref.end(), [](const Rec& x, const Rec& y) { return x.b < y.b; });
    turbosort::SortByKeyBuffer<Rec, uint64_t> rb(recs.size());
    CHECK(rb.capacity() >= recs.size());
    turbosort::sort_by_key_with_buffer(recs, rb, [](const Rec& r) { return (uint64_t)r.b; });
    for (size_t i = 0; i < recs.size(); ++i) CHECK(recs[i].id == ref[i].id);
    std::puts("ok");
    return 0;
}
