// Round trip of the learned coder's range coder over random symbol runs with
// 12-bit and small uniform frequency tables (built and run by
// tests/test_learned_cpu.py).
#include <cstdio>
#include <random>
#include <vector>
#include "learned_model.hpp"
using namespace curc::learned;
int main() {
    std::mt19937 rng(7);
    for (int trial = 0; trial < 200; ++trial) {
        int n = 1 + rng() % 20000;
        std::vector<std::vector<uint32_t>> fr(n);
        std::vector<int> sym(n);
        for (int i = 0; i < n; ++i) {
            int k = (rng() % 3 == 0) ? 1 + rng() % 320 : (rng() % 2 ? 4 : 16);
            uint32_t total = (k > 16 || rng() % 5 == 0) ? k : TOTAL;
            std::vector<uint32_t> f(k, 1);
            if (total == TOTAL) { uint32_t left = TOTAL - k; for (int j = 0; j < k && left; ++j) { uint32_t a = (j == k-1) ? left : rng() % (left + 1); f[j] += a; left -= a; } }
            fr[i] = f; sym[i] = rng() % k;
            if (rng() % 4 == 0) { int mx = 0; for (int j = 1; j < k; ++j) if (f[j] > f[mx]) mx = j; sym[i] = mx; }
        }
        RangeEncoder enc;
        for (int i = 0; i < n; ++i) { uint32_t cum = 0, tot = 0; for (int j = 0; j < (int)fr[i].size(); ++j) { if (j < sym[i]) cum += fr[i][j]; tot += fr[i][j]; } enc.encode(cum, fr[i][sym[i]], tot); }
        std::string s = enc.finish();
        RangeDecoder dec((const uint8_t*)s.data(), s.size());
        for (int i = 0; i < n; ++i) {
            uint32_t tot = 0; for (auto v : fr[i]) tot += v;
            uint32_t v = dec.peek(tot), cum = 0; int o = 0;
            while (cum + fr[i][o] <= v) cum += fr[i][o++];
            dec.consume(cum, fr[i][o]);
            if (o != sym[i]) { printf("mismatch trial %d at %d\n", trial, i); return 1; }
        }
    }
    printf("range coder round trips ok\n");
}
