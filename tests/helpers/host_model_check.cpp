// Test helper (CPU): the decoder's host form of the network
// (learned::model_freqs_host) gives the frequencies of the integer model
// (learned::model_freqs) on random anchors of random models with
// full-range int8 weights, in every form this CPU runs (int16 loops, and
// the AVX2 and AVX-512 VNNI byte dot products where the CPU has them).
#include <cstdio>
#include <random>
#include <vector>

#include "learned_model.hpp"

using namespace curc::learned;

int main() {
    std::mt19937_64 rng(21);
    auto uni = [&](int lo, int hi) { return int(std::uniform_int_distribution<int>(lo, hi)(rng)); };
    long long bad = 0;
    for (int trial = 0; trial < 4; ++trial) {
        static Model M;
        for (auto& r : M.w1)
            for (auto& w : r) w = int8_t(uni(-128, 127));
        for (auto& r : M.w2)
            for (auto& w : r) w = int8_t(uni(-128, 127));
        for (auto& r : M.w3)
            for (auto& w : r) w = int8_t(uni(-128, 127));
        for (auto& b : M.b1) b = uni(-500, 2000);
        for (auto& b : M.b2) b = uni(-20000, 200000);
        for (auto& b : M.b3) b = uni(-50000, 50000);
        M.m1 = uni(1, 8);
        M.sh1 = uni(2, 8);
        M.m2 = uni(1, 4);
        M.sh2 = uni(8, 14);
        M.zmul = 1 << uni(8, 13);
        for (int i = 0; i < LUTN; ++i) M.lut[i] = (65536u >> (i / 16)) | 1u;
        static HostModel H(M);
        H = HostModel(M);
        const int best = H.best_kind();
        for (int kind = HostModel::INT16; kind <= best; ++kind) {
            H.kind = kind;
            if (trial == 0) std::printf("form %d\n", kind);
            for (int a = 0; a < 20000; ++a) {
                int idx[24];
                const int n = uni(1, 24);
                for (int t = 0; t < n; ++t) idx[t] = uni(0, IN - 1);
                const int gmax = uni(0, 511);
                uint32_t fb[NB], fg[NG], hb[NB], hg[NG];
                model_freqs(M, idx, n, gmax, fb, fg);
                model_freqs_host(H, idx, n, gmax, hb, hg);
                for (int j = 0; j < NB; ++j) bad += fb[j] != hb[j];
                for (int j = 0; j < NG; ++j) bad += fg[j] != hg[j];
            }
        }
    }
    std::puts(bad ? "host model FAILED" : "host model ok");
    return bad ? 1 : 0;
}
