// Test helper (CPU): the learned mismatch stream written from the coding
// rules with the host integer model, then read back by the decoder the
// product uses for archives (learned::decode_stream).  Random model,
// pseudogenome and records; every offset and base must come back.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <random>
#include <string>
#include <vector>

#include "learned_model.hpp"

using namespace curc::learned;

int main() {
    std::mt19937_64 rng(11);
    auto uni = [&](int lo, int hi) { return int(std::uniform_int_distribution<int>(lo, hi)(rng)); };
    static Model M;
    for (auto& row : M.w1)
        for (auto& w : row) w = int8_t(uni(-20, 20));
    for (auto& row : M.w2)
        for (auto& w : row) w = int8_t(uni(-20, 20));
    for (auto& row : M.w3)
        for (auto& w : row) w = int8_t(uni(-20, 20));
    for (auto& b : M.b1) b = uni(-50, 200);
    for (auto& b : M.b2) b = uni(-2000, 20000);
    for (auto& b : M.b3) b = uni(-5000, 5000);
    M.m1 = 1;
    M.sh1 = 2;
    M.m2 = 1;
    M.sh2 = 12;
    M.zmul = 1 << 10;
    for (int i = 0; i < LUTN; ++i) {
        const double v = 65536.0 * std::exp(-double(i) / 16.0);
        M.lut[i] = v < 1 ? 1u : uint32_t(v);
    }
    int failures = 0;
    for (int L : {75, 150, 250}) {
        const uint64_t rl = 40000;
        std::string ref(rl, 'A');
        for (auto& c : ref) c = "ACGT"[uni(0, 3)];
        const size_t R = 40000;
        std::vector<uint64_t> pos(R);
        std::vector<uint8_t> strand(R), cnt(R);
        std::vector<std::vector<int>> offs(R);
        std::vector<std::string> bases(R);
        for (size_t r = 0; r < R; ++r) {
            pos[r] = uint64_t(uni(0, int(rl) - L));
            strand[r] = uint8_t(uni(0, 1));
            const int m = uni(0, 9) < 6 ? 0 : uni(1, 5);
            std::vector<int> o;
            while (int(o.size()) < m) {
                const int x = uni(0, L - 1);
                bool dup = false;
                for (int y : o) dup |= y == x;
                if (!dup) o.push_back(x);
            }
            std::sort(o.begin(), o.end());
            for (int x : o) {
                char b;
                do b = "ACGTN"[uni(0, 4)];
                while (b == ref[pos[r] + uint64_t(x)]);
                bases[r].push_back(b);
            }
            offs[r] = o;
            cnt[r] = uint8_t(m);
        }
        // write: chunks of CHUNK_RECORDS records with mismatches
        std::vector<std::string> chunks;
        RangeEncoder* enc = nullptr;
        BinModels* bins = nullptr;
        size_t in_chunk = 0;
        const uint8_t* g = reinterpret_cast<const uint8_t*>(ref.data());
        for (size_t r = 0; r < R; ++r) {
            const int m = cnt[r];
            if (!m) continue;
            if (!enc || in_chunk == CHUNK_RECORDS) {
                if (enc) chunks.push_back(enc->finish());
                delete enc;
                delete bins;
                enc = new RangeEncoder;
                bins = new BinModels;
                in_chunk = 0;
            }
            ++in_chunk;
            for (int j = 0; j <= m; ++j) {
                const int q = j == 0 ? -1 : offs[r][j - 1];
                const char prev = j >= 2 ? bases[r][j - 2] : 0;
                const int gmx = j < m ? L - 1 - q - (m - j) : 0;
                int idx[24];
                const int n = anchor_features(g, rl, pos[r], q, L, strand[r], prev, m - j, gmx, idx);
                uint32_t fb[NB], fg[NG];
                model_freqs(M, idx, n, gmx, fb, fg);
                if (j > 0) {
                    const int o = base_outcome(ref[pos[r] + uint64_t(q)], bases[r][j - 1]);
                    uint32_t cum = 0;
                    for (int t = 0; t < o; ++t) cum += fb[t];
                    enc->encode(cum, fb[o], TOTAL);
                }
                if (j < m) {
                    const int gap = offs[r][j] - q - 1;
                    const int gb = gap_bin(gap);
                    uint32_t cum = 0;
                    for (int t = 0; t < gb; ++t) cum += fg[t];
                    enc->encode(cum, fg[gb], TOTAL);
                    const int lo = gap_bin_lo(gb), hi = std::min(gap_bin_lo(gb + 1), gmx + 1);
                    const int bc = bin_context(q, L, strand[r]);
                    uint32_t oc, of, ot;
                    bins->lookup(bc, gb, gap - lo, hi - lo, oc, of, ot);
                    enc->encode(oc, of, ot);
                    bins->update(bc, gb, gap - lo);
                }
            }
        }
        if (enc) chunks.push_back(enc->finish());
        delete enc;
        delete bins;
        std::string s;
        const uint32_t nc = uint32_t(chunks.size());
        s.append(reinterpret_cast<const char*>(&nc), 4);
        for (auto& c : chunks) {
            const uint32_t len = uint32_t(c.size());
            s.append(reinterpret_cast<const char*>(&len), 4);
        }
        for (auto& c : chunks) s += c;
        // read back
        uint64_t total = 0;
        for (auto c : cnt) total += c;
        std::vector<uint16_t> off(total);
        std::vector<char> base(total);
        const std::string why = decode_stream(M, reinterpret_cast<const uint8_t*>(s.data()), s.size(), g, rl, L, R,
                                              pos.data(), strand.data(), cnt.data(), off.data(), base.data());
        size_t k = 0, bad = 0;
        for (size_t r = 0; r < R; ++r)
            for (int j = 0; j < cnt[r]; ++j, ++k) bad += off[k] != offs[r][j] || base[k] != bases[r][j];
        std::printf("L %d: %zu mismatches, %zu bytes, %zu wrong, %s\n", L, size_t(total), s.size(), bad,
                    why.empty() ? "decoded" : why.c_str());
        if (bad || !why.empty()) ++failures;
        // a corrupt stream must give an error or wrong values, never a crash
        std::string t = s;
        for (size_t i = 4 + 4 * chunks.size(); i < t.size(); i += 97) t[i] = char(t[i] ^ 0x5A);
        (void)decode_stream(M, reinterpret_cast<const uint8_t*>(t.data()), t.size(), g, rl, L, R, pos.data(),
                            strand.data(), cnt.data(), off.data(), base.data());
    }
    std::puts(failures ? "learned round trip FAILED" : "learned round trips ok");
    return failures ? 1 : 0;
}
