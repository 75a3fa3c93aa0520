// Test helper (CPU): curc::host::stable_order, the pair-position order of
// the paired-end position coder and decoder, against std::stable_sort on
// random keys (empty and one-element inputs, few distinct keys, constant
// keys, 32- and 64-bit keys, several thread counts, 2M keys).
#include <algorithm>
#include <cstdio>
#include <numeric>
#include <random>
#include <vector>

#include "host/stable_order.hpp"

template <class T>
static int check(size_t n, uint64_t range, int threads) {
    std::mt19937_64 rng(n * 31 + range);
    std::vector<T> key(n);
    for (auto& v : key) v = T(rng() % range);
    std::vector<uint32_t> ref(n);
    std::iota(ref.begin(), ref.end(), 0u);
    std::stable_sort(ref.begin(), ref.end(), [&](uint32_t a, uint32_t b) { return key[a] < key[b]; });
    const bool ok = curc::host::stable_order(key.data(), n, threads) == ref;
    if (!ok) std::printf("differs: n %zu range %llu threads %d\n", n, (unsigned long long)range, threads);
    return ok ? 0 : 1;
}

int main() {
    int bad = 0;
    bad += check<uint32_t>(0, 10, 16) + check<uint32_t>(1, 10, 16) + check<uint32_t>(1000, 7, 16);
    bad += check<uint32_t>(200000, 100, 3) + check<uint32_t>(150000, 1, 5);
    bad += check<uint64_t>(300000, 1ull << 40, 16) + check<uint64_t>(70000, 3, 2);
    bad += check<uint32_t>(2000000, 120000000, 16) + check<uint64_t>(2000000, 1ull << 33, 7);
    std::puts(bad ? "stable order FAILED" : "stable order ok");
    return bad;
}
