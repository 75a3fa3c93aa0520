// Learned mismatch coder: the integer model shared by the GPU encoder and the
// host decoder, and the range coder.  Everything that decides a probability
// is integer arithmetic (int8 weights, int32 accumulation, fixed-point
// requantisation, a table for the exponential), so both sides derive
// bit-identical 12-bit frequencies.
//
// What is coded, per record with mismatches (its count comes from the plain
// mismatch-count stream): walking the read in pseudogenome order from an
// anchor before its first base, the gap to the next mismatch (one of 16
// bins, then the offset inside the bin), then at that mismatch the read's base (one
// of the three other bases or N), and so on.  The network sees, at an
// anchor: the 16 pseudogenome bases around it, the position along the
// sequenced read (16 bins), whether it is the start anchor, and the previous
// mismatch's read base, and how many mismatches of the read are still to
// come.  The offset inside a gap bin is coded with adaptive per-bin
// frequencies.
#pragma once
#include <cstdint>
#include <algorithm>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#ifdef __CUDACC__
#define LM_HD __host__ __device__ __forceinline__
#else
#define LM_HD inline
#endif

namespace curc {
namespace learned {

constexpr int IN = 128;      // input features (one-hots, zero padded)
constexpr int HID = 128;     // hidden units per layer
constexpr int NB = 4;        // base outcomes: the three other bases, then N
constexpr int NG = 16;       // gap bins
constexpr int OUT = NB + NG;
constexpr int CTX = 16;      // pseudogenome bases around an anchor
constexpr int LUTN = 256;    // exponential table entries
constexpr uint32_t TOTAL = 4096;  // frequency total (12 bits)

// Gap bins: [lo, lo + width) with widths 1,1,1,1,2,2,4,4,8,8,16,16,32,32,64,320
// (gaps of reads up to 512 bases).
LM_HD int gap_bin_lo(int b) {
    constexpr int lo[NG + 1] = {0, 1, 2, 3, 4, 6, 8, 12, 16, 24, 32, 48, 64, 96, 128, 192, 512};
    return lo[b];
}
LM_HD int gap_bin(int g) {
    int b = 0;
    while (b + 1 < NG && g >= gap_bin_lo(b + 1)) ++b;
    return b;
}

// Base outcome of read base rb at pseudogenome base gb (ASCII): index among
// the three other bases in A<C<G<T order, or 3 for N; -1 if not a mismatch.
LM_HD int base_outcome(char gb, char rb) {
    if (rb == 'N') return 3;
    const char order[4] = {'A', 'C', 'G', 'T'};
    int k = 0;
    for (int t = 0; t < 4; ++t) {
        if (order[t] == gb) continue;
        if (order[t] == rb) return k;
        ++k;
    }
    return -1;
}
LM_HD char outcome_base(char gb, int o) {
    if (o == 3) return 'N';
    const char order[4] = {'A', 'C', 'G', 'T'};
    int k = 0;
    for (int t = 0; t < 4; ++t) {
        if (order[t] == gb) continue;
        if (k == o) return order[t];
        ++k;
    }
    return '?';
}

LM_HD int code_of(char c) {
    switch (c) {
        case 'A': return 0;
        case 'C': return 1;
        case 'G': return 2;
        case 'T': return 3;
        default: return -1;
    }
}

// Active input features of an anchor (indices of the ones), at most 20.
// gmax: largest gap that can follow the anchor (when a mismatch is still to
// come).
// ref/rl: pseudogenome (ASCII) and its length; rpos: the record's position;
// q: anchor offset in pseudogenome order (-1 for the start anchor); L, strand;
// prev: previous mismatch's read base (0 if none); remaining: mismatches of
// the read still to come after this anchor (its count is known to both
// sides from the mismatch-count stream).
LM_HD int anchor_features(const uint8_t* ref, uint64_t rl, uint64_t rpos, int q, int L, int strand, char prev,
                          int remaining, int gmax, int* idx) {
    int n = 0;
    for (int t = 0; t < CTX; ++t) {
        const int64_t p = int64_t(rpos) + q - CTX / 2 + t;
        if (p < 0 || uint64_t(p) >= rl) continue;
        const int c = code_of(char(ref[p]));
        if (c >= 0) idx[n++] = 4 * t + c;
    }
    if (q < 0) {
        idx[n++] = 80;  // start anchor
    } else {
        const int rq = strand ? L - 1 - q : q;  // position along the sequenced read
        idx[n++] = 64 + (rq * 16) / L;
    }
    const int pc = prev == 'N' ? 4 : code_of(prev);
    if (pc >= 0) idx[n++] = 81 + pc;
    idx[n++] = 86 + (remaining < 4 ? remaining : 4);
    if (remaining > 0) idx[n++] = 96 + gap_bin(gmax);  // the last gap bin that can occur
    return n;
}

// Integer model.  acc1 = W1[:, active] summed + b1; a1 = clamp((acc1*m1 +
// round) >> sh1, 0, 127); the same for layer 2; z = W3 a2 + b3.
struct Model {
    int8_t w1[HID][IN];
    int32_t b1[HID];
    int8_t w2[HID][HID];
    int32_t b2[HID];
    int8_t w3[OUT][HID];
    int32_t b3[OUT];
    int32_t m1, sh1, m2, sh2;   // requantisation multipliers and shifts
    int32_t zmul;               // logit difference -> table index (16.16)
    uint32_t lut[LUTN];         // exp(-i/16) * 2^16, at least 1
};

LM_HD int32_t requant(int32_t acc, int32_t m, int32_t sh) {
    if (acc <= 0) return 0;
    const int64_t v = (int64_t(acc) * m + (int64_t(1) << (sh - 1))) >> sh;
    return v > 127 ? 127 : int32_t(v);
}

// Frequencies (total TOTAL) of the first `k` outcomes from their logits,
// each >= 1; outcomes k .. n-1 cannot occur and get 0.  `lut` and `zmul`
// are the model's exponential table and logit scale.
LM_HD void logits_to_freq_lut(const uint32_t* lut, int32_t zmul, const int32_t* z, int k, int n, uint32_t* f) {
    for (int j = k; j < n; ++j) f[j] = 0;
    int32_t mx = z[0];
    int am = 0;
    for (int j = 1; j < k; ++j)
        if (z[j] > mx) {
            mx = z[j];
            am = j;
        }
    uint64_t tot = 0;
    uint32_t e[NG];
    for (int j = 0; j < k; ++j) {
        const int64_t d = int64_t(mx) - z[j];
        int64_t i = (d * zmul) >> 16;
        if (i > LUTN - 1) i = LUTN - 1;
        e[j] = lut[i];
        tot += e[j];
    }
    uint32_t sum = 0;
    for (int j = 0; j < k; ++j) {
        f[j] = 1 + uint32_t((uint64_t(e[j]) * (TOTAL - uint32_t(k))) / tot);
        sum += f[j];
    }
    f[am] += TOTAL - sum;
}

LM_HD void logits_to_freq(const Model& M, const int32_t* z, int k, int n, uint32_t* f) {
    logits_to_freq_lut(M.lut, M.zmul, z, k, n, f);
}

// The network at one anchor: base and gap frequencies (gap bins beyond the
// one holding gmax get 0).
LM_HD void model_freqs(const Model& M, const int* idx, int nidx, int gmax, uint32_t* fb, uint32_t* fg) {
    int32_t a1[HID], a2[HID];
    for (int h = 0; h < HID; ++h) {
        int32_t acc = M.b1[h];
        for (int t = 0; t < nidx; ++t) acc += M.w1[h][idx[t]];
        a1[h] = requant(acc, M.m1, M.sh1);
    }
    for (int h = 0; h < HID; ++h) {
        int32_t acc = M.b2[h];
        for (int t = 0; t < HID; ++t) acc += int32_t(M.w2[h][t]) * a1[t];
        a2[h] = requant(acc, M.m2, M.sh2);
    }
    int32_t z[OUT];
    for (int o = 0; o < OUT; ++o) {
        int32_t acc = M.b3[o];
        for (int t = 0; t < HID; ++t) acc += int32_t(M.w3[o][t]) * a2[t];
        z[o] = acc;
    }
    logits_to_freq(M, z, NB, NB, fb);
    logits_to_freq(M, z + NB, gap_bin(gmax < 0 ? 0 : gmax) + 1, NG, fg);
}

// Host form of the network for the decoder, which evaluates it once per
// anchor: the weights widened to int16 once (layer 1 transposed, so an
// anchor's active inputs add whole rows) so that the products vectorise
// (16-bit multiply-add).  The activations after requant lie in [0, 127], so
// every product and sum is the int32 value model_freqs computes, and
// integer sums are exact in any order: the frequencies are model_freqs's.
//
// On x86-64 hosts with AVX2 or AVX-512 VNNI, layers 2 and 3 run on the
// unsigned-by-signed byte dot-product instructions instead (chosen once, at
// run time, from what the CPU reports): the activations, in [0, 127], are
// the unsigned bytes and the int8 weights the signed ones, stored in groups
// of four inputs per output.  VPDPBUSD sums four exact products into int32;
// VPMADDUBSW sums two into int16, which cannot saturate here (|2 x 127 x
// 128| < 2^15), before VPMADDWD widens them.  A model whose requantisation
// multipliers are not positive (activations could then be negative) keeps
// the int16 loops.
#if !defined(__CUDACC__) && defined(__x86_64__) && defined(__GNUC__)
#define LM_HOST_X86 1
#include <immintrin.h>
#endif

constexpr int OUT_PAD = 32;  // layer-3 outputs padded to two 16-lane groups

// The host form and the decoder that uses it have internal linkage: their
// bodies depend on the compiler (the CUDA compiler's copy keeps the int16
// loops), so no translation unit may share another's copy.
namespace {

struct HostModel {
    enum Kind { INT16 = 0, AVX2 = 1, VNNI512 = 2 };
    const Model* M;
    int kind = INT16;
    alignas(64) int16_t w1t[IN][HID];
    alignas(64) int16_t w2[HID][HID];
    alignas(64) int16_t w3[OUT][HID];
    alignas(64) int8_t w2q[HID / 4][HID][4];      // [input group][output][input in group]
    alignas(64) int8_t w3q[HID / 4][OUT_PAD][4];  // the same, outputs past OUT zero
    explicit HostModel(const Model& m) : M(&m) {
        for (int h = 0; h < HID; ++h)
            for (int i = 0; i < IN; ++i) w1t[i][h] = m.w1[h][i];
        for (int h = 0; h < HID; ++h)
            for (int t = 0; t < HID; ++t) w2[h][t] = m.w2[h][t];
        for (int o = 0; o < OUT; ++o)
            for (int t = 0; t < HID; ++t) w3[o][t] = m.w3[o][t];
        std::memset(w3q, 0, sizeof(w3q));
        for (int t = 0; t < HID; ++t) {
            for (int h = 0; h < HID; ++h) w2q[t / 4][h][t % 4] = m.w2[h][t];
            for (int o = 0; o < OUT; ++o) w3q[t / 4][o][t % 4] = m.w3[o][t];
        }
        kind = best_kind();
    }
    // The fastest form this CPU runs for this model.
    int best_kind() const {
        if (M->m1 <= 0 || M->m2 <= 0) return INT16;
#ifdef LM_HOST_X86
        __builtin_cpu_init();
        if (__builtin_cpu_supports("avx512f") && __builtin_cpu_supports("avx512bw") &&
            __builtin_cpu_supports("avx512dq") && __builtin_cpu_supports("avx512vl") &&
            __builtin_cpu_supports("avx512vnni"))
            return VNNI512;
        if (__builtin_cpu_supports("avx2")) return AVX2;
#endif
        return INT16;
    }
};

#ifdef LM_HOST_X86
// acc[o] = sum over t of a[t] * wq[t/4][o][t%4], for o < 16*groups16, t < HID
// (a: HID unsigned bytes; acc: int32, overwritten).
__attribute__((target("avx512f,avx512bw,avx512vnni"))) inline void dot_u8s8_vnni512(const int8_t* wq, int outs,
                                                                                    const uint8_t* a, int32_t* acc) {
    const int groups16 = outs / 16;
    __m512i s[HID / 16];
    for (int c = 0; c < groups16; ++c) s[c] = _mm512_setzero_si512();
    for (int g = 0; g < HID / 4; ++g) {
        int32_t four;
        std::memcpy(&four, a + 4 * g, 4);
        const __m512i x = _mm512_set1_epi32(four);
        const int8_t* row = wq + size_t(g) * outs * 4;
        for (int c = 0; c < groups16; ++c)
            s[c] = _mm512_dpbusd_epi32(s[c], x, _mm512_load_si512(reinterpret_cast<const void*>(row + 64 * c)));
    }
    for (int c = 0; c < groups16; ++c) _mm512_storeu_si512(reinterpret_cast<void*>(acc + 16 * c), s[c]);
}

__attribute__((target("avx2"))) inline void dot_u8s8_avx2(const int8_t* wq, int outs, const uint8_t* a,
                                                           int32_t* acc) {
    const __m256i ones = _mm256_set1_epi16(1);
    for (int c0 = 0; c0 < outs; c0 += 64) {  // 64 outputs (8 registers) at a time
        __m256i s[8];
        const int nc = std::min(8, (outs - c0) / 8);
        for (int c = 0; c < nc; ++c) s[c] = _mm256_setzero_si256();
        for (int g = 0; g < HID / 4; ++g) {
            int32_t four;
            std::memcpy(&four, a + 4 * g, 4);
            const __m256i x = _mm256_set1_epi32(four);
            const int8_t* row = wq + (size_t(g) * outs + c0) * 4;
            for (int c = 0; c < nc; ++c) {
                const __m256i w = _mm256_load_si256(reinterpret_cast<const __m256i*>(row + 32 * c));
                s[c] = _mm256_add_epi32(s[c], _mm256_madd_epi16(_mm256_maddubs_epi16(x, w), ones));
            }
        }
        for (int c = 0; c < nc; ++c) _mm256_storeu_si256(reinterpret_cast<__m256i*>(acc + c0 + 8 * c), s[c]);
    }
}
#endif

// The network at one anchor in form KIND.  Always inlined into the wrappers
// below, so that its plain loops (layer 1, the requantisations) are
// vectorised for the instruction set of the wrapper's form.
template <int KIND>
__attribute__((always_inline)) inline void host_freqs(const HostModel& H, const int* idx, int nidx, int gmax,
                                                      uint32_t* fb, uint32_t* fg) {
    const Model& M = *H.M;
    alignas(64) int32_t acc1[HID];
    for (int h = 0; h < HID; ++h) acc1[h] = M.b1[h];
    for (int t = 0; t < nidx; ++t) {
        const int16_t* row = H.w1t[idx[t]];
#pragma omp simd
        for (int h = 0; h < HID; ++h) acc1[h] += row[h];
    }
    int32_t z[OUT];
    if constexpr (KIND == HostModel::INT16) {
        alignas(64) int16_t a1[HID], a2[HID];
        for (int h = 0; h < HID; ++h) a1[h] = int16_t(requant(acc1[h], M.m1, M.sh1));
        for (int h = 0; h < HID; ++h) {
            int32_t acc = 0;
            const int16_t* w = H.w2[h];
#pragma omp simd reduction(+ : acc)
            for (int t = 0; t < HID; ++t) acc += int32_t(w[t]) * int32_t(a1[t]);
            a2[h] = int16_t(requant(acc + M.b2[h], M.m2, M.sh2));
        }
        for (int o = 0; o < OUT; ++o) {
            int32_t acc = 0;
            const int16_t* w = H.w3[o];
#pragma omp simd reduction(+ : acc)
            for (int t = 0; t < HID; ++t) acc += int32_t(w[t]) * int32_t(a2[t]);
            z[o] = acc + M.b3[o];
        }
    }
#ifdef LM_HOST_X86
    else {
        alignas(64) uint8_t u1[HID], u2[HID];
        alignas(64) int32_t acc[HID > OUT_PAD ? HID : OUT_PAD];
#pragma omp simd
        for (int h = 0; h < HID; ++h) u1[h] = uint8_t(requant(acc1[h], M.m1, M.sh1));
        if constexpr (KIND == HostModel::VNNI512)
            dot_u8s8_vnni512(&H.w2q[0][0][0], HID, u1, acc);
        else
            dot_u8s8_avx2(&H.w2q[0][0][0], HID, u1, acc);
#pragma omp simd
        for (int h = 0; h < HID; ++h) u2[h] = uint8_t(requant(acc[h] + M.b2[h], M.m2, M.sh2));
        if constexpr (KIND == HostModel::VNNI512)
            dot_u8s8_vnni512(&H.w3q[0][0][0], OUT_PAD, u2, acc);
        else
            dot_u8s8_avx2(&H.w3q[0][0][0], OUT_PAD, u2, acc);
        for (int o = 0; o < OUT; ++o) z[o] = acc[o] + M.b3[o];
    }
#endif
    logits_to_freq(M, z, NB, NB, fb);
    logits_to_freq(M, z + NB, gap_bin(gmax < 0 ? 0 : gmax) + 1, NG, fg);
}

#ifdef LM_HOST_X86
__attribute__((target("avx512f,avx512bw,avx512dq,avx512vl,avx512vnni"))) inline void host_freqs_vnni512(
    const HostModel& H, const int* idx, int nidx, int gmax, uint32_t* fb, uint32_t* fg) {
    host_freqs<HostModel::VNNI512>(H, idx, nidx, gmax, fb, fg);
}
__attribute__((target("avx2"))) inline void host_freqs_avx2(const HostModel& H, const int* idx, int nidx, int gmax,
                                                             uint32_t* fb, uint32_t* fg) {
    host_freqs<HostModel::AVX2>(H, idx, nidx, gmax, fb, fg);
}
#endif

inline void model_freqs_host(const HostModel& H, const int* idx, int nidx, int gmax, uint32_t* fb, uint32_t* fg) {
#ifdef LM_HOST_X86
    if (H.kind == HostModel::VNNI512) return host_freqs_vnni512(H, idx, nidx, gmax, fb, fg);
    if (H.kind == HostModel::AVX2) return host_freqs_avx2(H, idx, nidx, gmax, fb, fg);
#endif
    host_freqs<HostModel::INT16>(H, idx, nidx, gmax, fb, fg);
}

}  // namespace

// Context of the adaptive in-bin models.  One context: splitting them by
// strand and read position (16 contexts) spread the 16384-record chunks too
// thin and coded 1% larger on the ramped-error workload.
constexpr int BIN_CTX = 1;
LM_HD int bin_context(int, int, int) { return 0; }

// Adaptive frequencies of the offset inside each gap bin (the network gives
// the bin), one set per bin context: reset at the start of each
// independently coded chunk, updated after every coded gap in the same way
// by the encoder and the decoder.
class BinModels {
public:
    static constexpr uint32_t INC = 24, LIMIT = 1u << 15;
    BinModels() {
        for (int c = 0; c < BIN_CTX; ++c)
            for (int b = 0; b < NG; ++b) {
                f_[c][b].assign(size_t(gap_bin_lo(b + 1) - gap_bin_lo(b)), 1);
                tot_[c][b] = uint32_t(f_[c][b].size());
            }
    }
    // cumulative count, count and total of offset o among the first w offsets
    void lookup(int c, int b, int o, int w, uint32_t& cum, uint32_t& freq, uint32_t& total) const {
        cum = 0;
        total = 0;
        for (int j = 0; j < w; ++j) {
            if (j < o) cum += f_[c][b][j];
            total += f_[c][b][j];
        }
        freq = f_[c][b][o];
    }
    // offset whose cumulative range holds v, among the first w offsets
    int find(int c, int b, int w, uint32_t v, uint32_t& cum, uint32_t& freq) const {
        cum = 0;
        int o = 0;
        while (o + 1 < w && cum + f_[c][b][o] <= v) cum += f_[c][b][o++];
        freq = f_[c][b][o];
        return o;
    }
    uint32_t total(int c, int b, int w) const {
        uint32_t t = 0;
        for (int j = 0; j < w; ++j) t += f_[c][b][j];
        return t;
    }
    void update(int c, int b, int o) {
        f_[c][b][o] += INC;
        tot_[c][b] += INC;
        if (tot_[c][b] > LIMIT) {
            tot_[c][b] = 0;
            for (auto& x : f_[c][b]) {
                x = (x + 1) / 2;
                tot_[c][b] += x;
            }
        }
    }

private:
    std::vector<uint32_t> f_[BIN_CTX][NG];
    uint32_t tot_[BIN_CTX][NG];
};

// ------------------------------------------------------------ range coder
// Carry-propagating range coder (32-bit range, 64-bit low with a cached
// byte, as in LZMA's), symbols given as (cumulative, frequency, total).
class RangeEncoder {
public:
    void encode(uint32_t cum, uint32_t freq, uint32_t total) {
        const uint32_t r = range_ / total;
        low_ += uint64_t(r) * cum;
        range_ = r * freq;
        while (range_ < (1u << 24)) {
            range_ <<= 8;
            shift_low();
        }
    }
    std::string finish() {
        for (int i = 0; i < 5; ++i) shift_low();
        return out_;
    }

private:
    void shift_low() {
        if (uint32_t(low_) < 0xFF000000u || (low_ >> 32) != 0) {
            const uint8_t carry = uint8_t(low_ >> 32);
            if (have_cache_) out_.push_back(char(uint8_t(cache_ + carry)));
            for (; pending_ > 0; --pending_) out_.push_back(char(uint8_t(0xFF + carry)));
            cache_ = uint8_t(low_ >> 24);
            have_cache_ = true;
        } else {
            ++pending_;
        }
        low_ = (low_ & 0x00FFFFFFu) << 8;
    }
    uint64_t low_ = 0;
    uint32_t range_ = 0xFFFFFFFFu;
    uint8_t cache_ = 0;
    bool have_cache_ = false;
    uint64_t pending_ = 0;
    std::string out_;
};

class RangeDecoder {
public:
    RangeDecoder(const uint8_t* p, size_t n) : p_(p), n_(n) {
        for (int i = 0; i < 4; ++i) code_ = (code_ << 8) | next();
    }
    // the cumulative count the next symbol falls in
    uint32_t peek(uint32_t total) {
        r_ = range_ / total;
        const uint32_t v = code_ / r_;
        return v < total ? v : total - 1;
    }
    void consume(uint32_t cum, uint32_t freq) {
        code_ -= r_ * cum;
        range_ = r_ * freq;
        while (range_ < (1u << 24)) {
            range_ <<= 8;
            code_ = (code_ << 8) | next();
        }
    }

private:
    uint8_t next() { return i_ < n_ ? p_[i_++] : 0; }
    const uint8_t* p_;
    size_t n_, i_ = 0;
    uint32_t code_ = 0, range_ = 0xFFFFFFFFu, r_ = 1;
};

// ------------------------------------------------------------ stream decoder
// Records with mismatches are coded in chunks of this many records, each
// chunk an independent range-coded stream (so chunks code and decode in
// parallel).  Stream layout: u32 chunk count, u32 byte length per chunk,
// then the chunks.
constexpr size_t CHUNK_RECORDS = 16384;

namespace {

// Decodes a learned stream.  Records come in emission order with their
// position on the main pseudogenome `ref` (ASCII, length rl), strand and
// mismatch count; the mismatches of record r are written from index first[r]
// = (counts of the records before it) on: their offsets along the read in
// pseudogenome order, and the read bases.  Returns an error message, empty
// when the stream decoded completely and consistently.
inline std::string decode_stream(const Model& M, const uint8_t* p, size_t bytes, const uint8_t* ref, uint64_t rl,
                                 int L, size_t records, const uint64_t* pos, const uint8_t* strand,
                                 const uint8_t* cnt, uint16_t* off, char* base) {
    std::vector<uint32_t> rlist;
    std::vector<uint64_t> first;
    uint64_t acc = 0;
    for (size_t r = 0; r < records; ++r) {
        if (cnt[r]) {
            if (pos[r] > rl || uint64_t(L) > rl - pos[r]) return "a record lies outside the pseudogenome";
            rlist.push_back(uint32_t(r));
            first.push_back(acc);
        }
        acc += cnt[r];
    }
    if (bytes < 4) return "short learned stream";
    uint32_t nc;
    std::memcpy(&nc, p, 4);
    const uint64_t expect = (rlist.size() + CHUNK_RECORDS - 1) / CHUNK_RECORDS;
    if (nc != expect && !(nc == 1 && rlist.empty())) return "learned stream: chunk count disagrees with the records";
    if (bytes < 4 + 4ull * nc) return "short learned stream";
    std::vector<uint64_t> coff(size_t(nc) + 1);
    coff[0] = 4 + 4ull * nc;
    for (uint32_t c = 0; c < nc; ++c) {
        uint32_t len;
        std::memcpy(&len, p + 4 + 4 * size_t(c), 4);
        coff[c + 1] = coff[c] + len;
    }
    if (coff[nc] != bytes) return "learned stream: length disagrees with its chunks";
    int bad = 0;
    const auto H = std::make_unique<HostModel>(M);
#pragma omp parallel for schedule(dynamic) reduction(+ : bad)
    for (int c = 0; c < int(nc); ++c) {
        RangeDecoder dec(p + coff[c], size_t(coff[c + 1] - coff[c]));
        BinModels bins;
        const size_t r0 = size_t(c) * CHUNK_RECORDS, r1 = std::min(rlist.size(), r0 + CHUNK_RECORDS);
        for (size_t ri = r0; ri < r1 && !bad; ++ri) {
            const size_t r = rlist[ri];
            const int m = cnt[r];
            int q = -1;
            char prev = 0;
            for (int j = 0; j <= m; ++j) {
                int idx[24];
                const int gmx = j < m ? L - 1 - q - (m - j) : 0;
                if (j < m && gmx < 0) {
                    ++bad;
                    break;
                }
                const int n = anchor_features(ref, rl, pos[r], q, L, strand[r], prev, m - j, gmx, idx);
                uint32_t fb[NB], fg[NG];
                model_freqs_host(*H, idx, n, gmx, fb, fg);
                if (j > 0) {
                    const uint32_t v = dec.peek(TOTAL);
                    uint32_t cum = 0;
                    int o = 0;
                    while (o < NB - 1 && cum + fb[o] <= v) cum += fb[o++];
                    dec.consume(cum, fb[o]);
                    prev = outcome_base(char(ref[pos[r] + uint64_t(q)]), o);
                    base[first[ri] + uint64_t(j - 1)] = prev;
                }
                if (j < m) {
                    uint32_t v = dec.peek(TOTAL), cum = 0;
                    int gb = 0;
                    while (gb < NG - 1 && cum + fg[gb] <= v) cum += fg[gb++];
                    if (!fg[gb]) {
                        ++bad;
                        break;
                    }
                    dec.consume(cum, fg[gb]);
                    const int lo = gap_bin_lo(gb), hi = std::min(gap_bin_lo(gb + 1), gmx + 1);
                    const int w = hi - lo > 1 ? hi - lo : 1;
                    const int bc = bin_context(q, L, strand[r]);
                    uint32_t oc, of;
                    const uint32_t ov = dec.peek(bins.total(bc, gb, w));
                    const int o = bins.find(bc, gb, w, ov, oc, of);
                    dec.consume(oc, of);
                    bins.update(bc, gb, o);
                    const int g = lo + o;
                    q = q + 1 + g;
                    if (q > L - 1) {
                        ++bad;
                        break;
                    }
                    off[first[ri] + uint64_t(j)] = uint16_t(q);
                }
            }
        }
    }
    return bad ? "learned stream does not decode consistently" : "";
}

}  // namespace

}  // namespace learned
}  // namespace curc
