// Stable order of indices by an unsigned key, on host threads.
//
// stable_order(key, n)[q] is the index i of the q-th smallest key, ties in
// ascending i: the permutation std::stable_sort(ids, key[a] < key[b]) gives
// (a stable order is unique).  LSD radix over the key's bytes, skipping the
// bytes in which all keys agree; each pass counts the digits of every
// thread's contiguous chunk, places each chunk after the same digit's items
// of the chunks before it, and scatters the chunks in order, so equal keys
// keep their index order.  The threads are std::threads, one per chunk, so
// every chunk has its worker whatever the caller's threading.
#pragma once
#include <algorithm>
#include <array>
#include <cstdint>
#include <thread>
#include <vector>

namespace curc {
namespace host {

// Chunks of [0, n) for up to `threads` threads (at least 65536 items each).
inline size_t chunk_count(size_t n, int threads) {
    return std::max<size_t>(1, std::min<size_t>(size_t(std::max(1, threads)), n / 65536 + 1));
}

// f(lo, hi, t) on each of the `nt` contiguous chunks of [0, n), one
// std::thread per chunk (the calling thread takes chunk 0).
template <class F>
void each_chunk(size_t n, size_t nt, F&& f) {
    const size_t chunk = (n + nt - 1) / nt;
    std::vector<std::thread> th;
    for (size_t t = 1; t < nt; ++t)
        th.emplace_back([&, t] { f(std::min(n, t * chunk), std::min(n, (t + 1) * chunk), t); });
    f(size_t(0), std::min(n, chunk), size_t(0));
    for (auto& x : th) x.join();
}

template <class T>
std::vector<uint32_t> stable_order(const T* key, size_t n, int threads = 16) {
    static_assert(sizeof(T) <= 8, "keys of at most 64 bits");
    std::vector<uint32_t> idx(n);
    for (size_t i = 0; i < n; ++i) idx[i] = uint32_t(i);
    if (n < 2) return idx;
    const size_t nt = chunk_count(n, threads);
    auto each = [&](auto&& f) { each_chunk(n, nt, f); };
    std::vector<T> k(key, key + n), k2(n);
    std::vector<uint32_t> idx2(n);
    // bytes in which some keys differ
    std::vector<uint64_t> dpart(nt, 0);
    each([&](size_t lo, size_t hi, size_t t) {
        uint64_t d = 0;
        for (size_t i = lo; i < hi; ++i) d |= uint64_t(k[i] ^ k[0]);
        dpart[t] = d;
    });
    uint64_t diff = 0;
    for (uint64_t d : dpart) diff |= d;
    std::vector<std::array<size_t, 256>> cnt(nt);
    for (int b = 0; b < int(sizeof(T)); ++b) {
        if (((diff >> (8 * b)) & 0xFF) == 0) continue;
        const int sh = 8 * b;
        each([&](size_t lo, size_t hi, size_t t) {
            auto& c = cnt[t];
            c.fill(0);
            for (size_t i = lo; i < hi; ++i) ++c[size_t(k[i] >> sh) & 0xFF];
        });
        size_t acc = 0;
        for (size_t d = 0; d < 256; ++d)
            for (size_t t = 0; t < nt; ++t) {
                const size_t v = cnt[t][d];
                cnt[t][d] = acc;
                acc += v;
            }
        each([&](size_t lo, size_t hi, size_t t) {
            auto& c = cnt[t];
            for (size_t i = lo; i < hi; ++i) {
                const size_t p = c[size_t(k[i] >> sh) & 0xFF]++;
                k2[p] = k[i];
                idx2[p] = idx[i];
            }
        });
        k.swap(k2);
        idx.swap(idx2);
    }
    return idx;
}

}  // namespace host
}  // namespace curc
