// CPU oracle for the CURC pseudogenome path -- TEST INFRASTRUCTURE ONLY.
// Stage restatements of the reference's src/compress.cu (cited per function)
// under the canonical sequential semantics described in oracle.hpp.
#include "oracle.hpp"

#include <algorithm>
#include <cstring>
#include <numeric>
#include <stdexcept>

namespace oracle {

Params Params::derive(int L, bool po, bool pe) {
    // preprocess.cpp:295-313
    Params p;
    p.read_len = L;
    p.unit = (L + 31) / 32;
    p.max_off = L * 65 / 100;
    p.kmer_size = L < 89 ? 36 * L / 100 : 32;
    p.kmer_index_pos = L - p.kmer_size - p.max_off;
    p.max_mismatch = L / 5;
    p.preserve_order = po;
    p.paired_end = pe;
    return p;
}

// ---------------------------------------------------------------- helpers

uint64_t murmur64(uint64_t x) {  // util.cuh:82-89 (fmix64)
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdULL;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ULL;
    x ^= x >> 33;
    return x;
}

uint32_t hash_size_for(size_t items) {  // util.cuh:72-80
    uint32_t hs;
    int order = 24;
    do {
        hs = 1u << order;
        ++order;
    } while (order <= 31 && hs < items);
    return hs;
}

// Bases [off, off+nb) of a packed read (MSB-first, 2 bits per base) as an
// integer whose first base is most significant.  util.cuh:180-188.
uint64_t word_at(const uint64_t* r, uint64_t off, int nb) {
    uint64_t w = off >> 5;
    unsigned s = unsigned(off & 31) * 2;
    uint64_t v = r[w] << s;
    if (64 - s < unsigned(2 * nb)) v |= r[w + 1] >> (64 - s);
    return v >> (64 - 2 * nb);
}

// Same on a padded contiguous bit string (always reads the next word).
// util.cuh:189-195.
uint64_t word_unaligned(const uint64_t* r, uint64_t off, int nb) {
    uint64_t w = off >> 5;
    unsigned s = unsigned(off & 31) * 2;
    uint64_t v = r[w] << s;
    if (s) v |= r[w + 1] >> (64 - s);
    return v >> (64 - 2 * nb);
}

static inline int code_at(const uint64_t* r, uint64_t off) {
    return int((r[off >> 5] >> (62 - 2 * (off & 31))) & 3);
}

char base_at(const uint64_t* r, uint64_t off) { return "ACGT"[code_at(r, off)]; }

uint64_t revcomp_kmer(uint64_t kmer, int k) {  // util.cuh:220-226
    uint64_t out = 0;
    for (int i = 0; i < k; ++i) {
        out = (out << 2) | (3 - (kmer & 3));
        kmer >>= 2;
    }
    return out;
}

char comp_base(char b) {  // util.cuh:152-164
    switch (b) {
        case 'a': return 't';
        case 'A': return 'T';
        case 'c': return 'g';
        case 'C': return 'G';
        case 'g': return 'c';
        case 'G': return 'C';
        case 't': return 'a';
        case 'T': return 'A';
        default: return 'N';
    }
}

static inline int enc(char c) {  // base_encode_table & 3: ACGT/acgt -> 0..3, else 0
    switch (c) {
        case 'C': case 'c': return 1;
        case 'G': case 'g': return 2;
        case 'T': case 't': return 3;
        default: return 0;
    }
}

uint64_t kmer_from_ascii(const char* s, int k) {  // util.cuh:271-281
    uint64_t v = 0;
    for (int i = 0; i < k; ++i) v = (v << 2) | uint64_t(enc(s[i]));
    return v;
}

// ---------------------------------------------------------------- a1

void pack_reads(const char* seq, size_t n, int L, uint64_t* packed, uint8_t* has_n) {
    // compress.cu:2159-2174 (pack), preprocess.cpp:149-152 (N test: 'N' only)
    const int W = (L + 31) / 32;
    for (size_t i = 0; i < n; ++i) {
        uint64_t* out = packed + i * W;
        std::fill(out, out + W, 0);
        bool hn = false;
        for (int j = 0; j < L; ++j) {
            char c = seq[i * L + j];
            hn |= (c == 'N');
            out[j >> 5] |= uint64_t(enc(c)) << (62 - 2 * (j & 31));
        }
        has_n[i] = hn;
    }
}

// ---------------------------------------------------------------- a2

void sort_dedupe(const uint64_t* db, int W, std::vector<uint32_t>& ids,
                 uint32_t* next, uint32_t* prev, uint16_t* offset) {
    // compress.cu:1400-1420 (thrust::sort is a stable merge sort for a
    // user comparator; ties keep ascending id order)
    std::stable_sort(ids.begin(), ids.end(), [&](uint32_t a, uint32_t b) {
        return std::lexicographical_compare(db + size_t(a) * W, db + size_t(a) * W + W,
                                            db + size_t(b) * W, db + size_t(b) * W + W);
    });
    for (size_t i = 0; i + 1 < ids.size(); ++i) {
        if (std::equal(db + size_t(ids[i]) * W, db + size_t(ids[i]) * W + W, db + size_t(ids[i + 1]) * W)) {
            next[ids[i]] = ids[i + 1];
            prev[ids[i + 1]] = ids[i];
            offset[ids[i]] = 0;
        }
    }
}

// ---------------------------------------------------------------- a3 + a4

// Three-way compare of prefix read a[0, len) with read b[off, off+len).
static int cmp_shifted(const uint64_t* a, uint64_t aoff, const uint64_t* b, uint64_t boff, int len) {
    for (int j = 0; j < len; j += 32) {
        int nb = std::min(32, len - j);
        uint64_t x = word_at(a, aoff + j, nb), y = word_at(b, boff + j, nb);
        if (x < y) return -1;
        if (x > y) return 1;
    }
    return 0;
}

void overlap_link(const Params& p, const uint64_t* db, const std::vector<uint32_t>& sorted,
                  uint32_t* next, uint32_t* prev, uint16_t* offset, const OverlapControl* ctl, int threads) {
    const int W = p.unit, L = p.read_len, k = p.kmer_size, kip = p.kmer_index_pos;
    // compress.cu:1427-1438: prefix set (no duplicate predecessor) and suffix set
    std::vector<uint32_t> pre, suf;
    for (uint32_t id : sorted) {
        if (prev[id] == INVALID) pre.push_back(id);
        if (next[id] == INVALID) suf.push_back(id);
    }
    // compress.cu:1440-1471: bucket by hash of the k-mer at kmer_index_pos,
    // stable within a bucket (lexicographic order kept)
    const uint32_t mask = hash_size_for(pre.size()) - 1;
    std::vector<uint32_t> key(pre.size());
    for (size_t i = 0; i < pre.size(); ++i)
        key[i] = uint32_t(murmur64(word_at(db + size_t(pre[i]) * W, kip, k)) & mask);
    std::vector<uint32_t> ord(pre.size());
    std::iota(ord.begin(), ord.end(), 0);
    std::stable_sort(ord.begin(), ord.end(), [&](uint32_t a, uint32_t b) { return key[a] < key[b]; });
    std::vector<uint32_t> va(pre.size()), vk(pre.size());
    for (size_t i = 0; i < ord.size(); ++i) { va[i] = pre[ord[i]]; vk[i] = key[ord[i]]; }

    // compress.cu:1473-1532, one suffix at a time in list order
    for (int off = 1; off < p.max_off; ++off) {
        const int cl = L - off;
        // visiting order: this pass's picks that are still unlinked suffixes
        // (in the order given), then the rest in list order
        std::vector<uint32_t> order;
        if (ctl)
            for (const ContestPick& c : ctl->picks)
                if (c.pass == off && std::find(order.begin(), order.end(), c.suffix) == order.end() &&
                    std::find(suf.begin(), suf.end(), c.suffix) != suf.end())
                    order.push_back(c.suffix);
        const size_t npick = order.size();
        for (uint32_t s : suf)
            if (std::find(order.begin(), order.begin() + npick, s) == order.begin() + npick) order.push_back(s);
        std::vector<std::pair<uint32_t, uint32_t>> runs;  // (run, suffix) of suffixes with a matching prefix
        // the searches read only the prefix index and the reads, which no
        // link changes, so they run in parallel; the links below are made
        // one suffix at a time in the visiting order
        std::vector<size_t> los(order.size()), his(order.size());
#pragma omp parallel for schedule(dynamic, 1024) num_threads(threads)
        for (size_t i = 0; i < order.size(); ++i) {
            const uint64_t* sr = db + size_t(order[i]) * W;
            uint32_t h = uint32_t(murmur64(word_at(sr, kip + off, k)) & mask);
            auto rng = std::equal_range(vk.begin(), vk.end(), h);
            size_t lo = rng.first - vk.begin(), hi = rng.second - vk.begin();
            // lower bound of suffix[off, L) among prefix[0, cl)
            size_t cnt = hi - lo;
            while (cnt > 0) {
                size_t step = cnt / 2, it = lo + step;
                if (cmp_shifted(db + size_t(va[it]) * W, 0, sr, off, cl) < 0) {
                    lo = it + 1;
                    cnt -= step + 1;
                } else {
                    cnt = step;
                }
            }
            los[i] = lo;
            his[i] = hi;
        }
        for (size_t i = 0; i < order.size(); ++i) {
            const uint32_t s = order[i];
            const uint64_t* sr = db + size_t(s) * W;
            const size_t lo = los[i], hi = his[i];
            if (ctl && ctl->log && lo < hi && cmp_shifted(db + size_t(va[lo]) * W, 0, sr, off, cl) == 0)
                runs.push_back({uint32_t(lo), s});
            for (size_t q = lo; q < hi; ++q) {
                uint32_t pr = va[q];
                if (pr == s || prev[pr] != INVALID) continue;
                if (cmp_shifted(db + size_t(pr) * W, 0, sr, off, cl) == 0) {
                    prev[pr] = s;
                    next[s] = pr;
                    offset[s] = uint16_t(off);
                }
                break;
            }
        }
        if (ctl && ctl->log) {
            std::stable_sort(runs.begin(), runs.end(),
                             [](const auto& a, const auto& b) { return a.first < b.first; });
            for (size_t i = 0; i < runs.size();) {
                size_t j = i;
                while (j < runs.size() && runs[j].first == runs[i].first) ++j;
                if (j - i > 1)
                    for (size_t k = i; k < j; ++k)
                        ctl->log->push_back({uint32_t(off), runs[k].first, runs[k].second, next[runs[k].second]});
                i = j;
            }
        }
        std::vector<uint32_t> rem;
        rem.reserve(suf.size());
        for (uint32_t s : suf)
            if (next[s] == INVALID) rem.push_back(s);
        suf.swap(rem);
    }
}

// ---------------------------------------------------------------- a5

void chain_filter(size_t reads_count, const std::vector<uint32_t>& sorted,
                  uint32_t* next, uint32_t* prev, const uint16_t* offset,
                  std::vector<uint32_t>& ref_ids, std::vector<uint32_t>& unmatch_ids) {
    // compress.cu:1539-1572
    std::vector<uint8_t> res(reads_count, 1);
    for (size_t r = 0; r < reads_count; ++r) {
        if (next[r] != INVALID && prev[r] != INVALID) continue;
        if (next[r] != INVALID && offset[r] == 0) continue;
        if (prev[r] != INVALID && offset[prev[r]] == 0) continue;
        res[r] = 0;
    }
    // A link is removed iff either end is filtered out (order independent).
    for (size_t r = 0; r < reads_count; ++r) {
        if (res[r]) continue;
        if (next[r] != INVALID) { prev[next[r]] = INVALID; next[r] = INVALID; }
        if (prev[r] != INVALID) { next[prev[r]] = INVALID; prev[r] = INVALID; }
    }
    ref_ids.clear();
    unmatch_ids.clear();
    for (uint32_t id : sorted) (res[id] ? ref_ids : unmatch_ids).push_back(id);
}

// ---------------------------------------------------------------- a6

void full_match_packed(const Params& p, const uint64_t* db, std::vector<uint32_t> pre,
                       std::vector<uint32_t> suf, uint32_t* next, uint32_t* prev, uint16_t* offset) {
    // compress.cu:1003-1174
    const int W = p.unit, L = p.read_len;
    auto R = [&](uint32_t id) { return db + size_t(id) * W; };
    for (int off = 1; off < L; ++off) {
        // Re-sort suffixes by read[off, L): the reference's 4-way split on
        // base off-1 followed by stable merges equals a stable sort of the
        // current list (which is ordered by read[off-1, L)).
        std::stable_sort(suf.begin(), suf.end(), [&](uint32_t a, uint32_t b) {
            return cmp_shifted(R(a), off, R(b), off, L - off) < 0;
        });
        const int bpl = std::min(10, L - off);
        const int len = L - off;
        // bucket walk: prefixes keyed by read[0, bpl), suffixes by read[off, off+bpl)
        size_t pi0 = 0, si0 = 0;
        while (pi0 < pre.size() && si0 < suf.size()) {
            uint64_t bp = word_at(R(pre[pi0]), 0, bpl), bs = word_at(R(suf[si0]), off, bpl);
            if (bp < bs) { ++pi0; continue; }
            if (bs < bp) { ++si0; continue; }
            size_t pe = pi0, se = si0;
            while (pe < pre.size() && word_at(R(pre[pe]), 0, bpl) == bp) ++pe;
            while (se < suf.size() && word_at(R(suf[se]), off, bpl) == bs) ++se;
            // one bucket: two-pointer merge (compress.cu:1089-1160)
            size_t pi = pi0, si = si0;
            while (pi < pe && si < se) {
                uint32_t P = pre[pi], S = suf[si];
                int c = cmp_shifted(R(P), bpl, R(S), off + bpl, len - bpl);
                if (c > 0) { ++si; continue; }
                if (c < 0) { ++pi; continue; }
                if (P == S) {
                    size_t cur = pi;
                    int tmp = 1;
                    while (pi + 1 < pe) {
                        ++pi;
                        P = pre[pi];
                        // the reference only tests "prefix word > suffix word"
                        tmp = 0;
                        for (int i = bpl; i < len; i += 32) {
                            int nb = std::min(32, len - i);
                            if (word_at(R(P), i, nb) > word_at(R(S), i + off, nb)) { tmp = 1; break; }
                        }
                        if (tmp != 0) break;
                        if (P != S) break;
                        tmp = 1;
                    }
                    if (tmp != 0) {
                        pi = cur;
                        ++si;
                        continue;
                    }
                    P = pre[pi];
                    while (pi > cur) { pre[pi] = pre[pi - 1]; --pi; }
                    pre[pi] = P;
                }
                next[S] = P;
                prev[P] = S;
                ++pi;
                ++si;
            }
            pi0 = pe;
            si0 = se;
        }
        for (uint32_t s : suf)
            if (next[s] != INVALID) offset[s] = uint16_t(off);
        pre.erase(std::remove_if(pre.begin(), pre.end(), [&](uint32_t id) { return prev[id] != INVALID; }), pre.end());
        suf.erase(std::remove_if(suf.begin(), suf.end(), [&](uint32_t id) { return next[id] != INVALID; }), suf.end());
    }
}

// ---------------------------------------------------------------- a7

void full_match_ascii(const Params& p, const char* nr, std::vector<uint32_t> ids, size_t n_total,
                      std::vector<uint32_t>& next, std::vector<uint32_t>& prev, std::vector<uint16_t>& offset) {
    // compress.cu:1176-1347 (ids sorted in place by the caller's copy)
    const int L = p.read_len;
    auto S = [&](uint32_t id) { return nr + size_t(id) * L; };
    std::stable_sort(ids.begin(), ids.end(), [&](uint32_t a, uint32_t b) { return std::memcmp(S(a), S(b), L) < 0; });
    next.assign(n_total, INVALID);
    prev.assign(n_total, INVALID);
    offset.assign(n_total, INVALOFF);
    for (size_t i = 1; i < ids.size(); ++i) {
        if (std::memcmp(S(ids[i - 1]), S(ids[i]), L) == 0) {
            prev[ids[i]] = ids[i - 1];
            next[ids[i - 1]] = ids[i];
            offset[ids[i - 1]] = 0;
        }
    }
    std::vector<uint32_t> pre, suf;
    for (uint32_t id : ids) {
        if (prev[id] == INVALID) pre.push_back(id);
        if (next[id] == INVALID) suf.push_back(id);
    }
    static const char alpha[5] = {'A', 'C', 'G', 'N', 'T'};
    auto bucket_of = [&](const char* s, int bpl) {
        // rank of s[0, bpl) in base 5 over ACGNT; -1 if a symbol is outside
        long v = 0;
        for (int i = 0; i < bpl; ++i) {
            const char* f = std::find(alpha, alpha + 5, s[i]);
            if (f == alpha + 5) return -1L;
            v = v * 5 + (f - alpha);
        }
        return v;
    };
    for (int off = 1; off < L; ++off) {
        std::stable_sort(suf.begin(), suf.end(), [&](uint32_t a, uint32_t b) {
            return std::memcmp(S(a) + off, S(b) + off, L - off) < 0;
        });
        const int bpl = std::min(3, L - off);
        size_t pi0 = 0, si0 = 0;
        while (pi0 < pre.size() && si0 < suf.size()) {
            long bp = bucket_of(S(pre[pi0]), bpl), bs = bucket_of(S(suf[si0]) + off, bpl);
            if (bp < bs) { ++pi0; continue; }
            if (bs < bp) { ++si0; continue; }
            size_t pe = pi0, se = si0;
            while (pe < pre.size() && bucket_of(S(pre[pe]), bpl) == bp) ++pe;
            while (se < suf.size() && bucket_of(S(suf[se]) + off, bpl) == bs) ++se;
            if (bp < 0) { pi0 = pe; si0 = se; continue; }
            size_t pi = pi0, si = si0;
            while (pi < pe && si < se) {
                uint32_t P = pre[pi], Q = suf[si];
                int c = std::memcmp(S(P) + bpl, S(Q) + off + bpl, L - off - bpl);
                if (c > 0) { ++si; continue; }
                if (c < 0) { ++pi; continue; }
                if (P == Q) {
                    size_t cur = pi;
                    int tmp = 1;
                    while (pi + 1 < pe) {
                        ++pi;
                        P = pre[pi];
                        tmp = std::memcmp(S(P) + bpl, S(Q) + off + bpl, L - off - bpl);
                        if (tmp != 0) break;
                        if (P != Q) break;
                        tmp = 1;
                    }
                    if (tmp != 0) {
                        pi = cur;
                        ++si;
                        continue;
                    }
                    P = pre[pi];
                    while (pi > cur) { pre[pi] = pre[pi - 1]; --pi; }
                    pre[pi] = P;
                }
                next[Q] = P;
                prev[P] = Q;
                ++pi;
                ++si;
            }
            pi0 = pe;
            si0 = se;
        }
        for (uint32_t s : suf)
            if (next[s] != INVALID) offset[s] = uint16_t(off);
        pre.erase(std::remove_if(pre.begin(), pre.end(), [&](uint32_t id) { return prev[id] != INVALID; }), pre.end());
        suf.erase(std::remove_if(suf.begin(), suf.end(), [&](uint32_t id) { return next[id] != INVALID; }), suf.end());
    }
}

// ---------------------------------------------------------------- a8

template <class Emit>
static void walk_chains(const std::vector<uint32_t>& ids, const uint32_t* next, const uint32_t* prev,
                        const uint16_t* offset, size_t reads_count, Emit emit) {
    // compress.cu:107-165: linear chains from their head; cycles are cut
    // after the member with the largest offset, which is emitted last.
    std::vector<uint8_t> visit(reads_count, 0);
    for (uint32_t r : ids) {
        if (visit[r]) continue;
        uint32_t i = r;
        while (prev[i] != INVALID && prev[i] != r) i = prev[i];
        if (prev[i] == r) {
            uint16_t mo = offset[i];
            uint32_t mid = i;
            while (i != r) {
                visit[i] = 1;
                i = next[i];
                if (offset[i] > mo) { mo = offset[i]; mid = i; }
            }
            visit[r] = 1;
            for (uint32_t s = next[mid]; s != mid; s = next[s]) emit(s, false);
            emit(mid, true);
        } else {
            while (next[i] != INVALID) {
                visit[i] = 1;
                emit(i, false);
                i = next[i];
            }
            visit[i] = 1;
            emit(i, true);
        }
    }
}

void assemble_packed(const uint64_t* db, int L, int W, const std::vector<uint32_t>& ids,
                     const uint32_t* next, const uint32_t* prev, const uint16_t* offset,
                     size_t reads_count, Pseudogenome& out) {
    walk_chains(ids, next, prev, offset, reads_count, [&](uint32_t id, bool tail) {
        out.records.push_back({id, 0, 0, out.seq.size()});
        int n = tail ? L : offset[id];
        const uint64_t* r = db + size_t(id) * W;
        for (int j = 0; j < n; ++j) out.seq.push_back(base_at(r, j));
    });
}

void assemble_ascii(const char* nr, int L, const std::vector<uint32_t>& ids,
                    const uint32_t* next, const uint32_t* prev, const uint16_t* offset,
                    size_t reads_count, Pseudogenome& out) {
    // compress.cu:167-217
    walk_chains(ids, next, prev, offset, reads_count, [&](uint32_t id, bool tail) {
        out.records.push_back({id, 1, 0, out.seq.size()});
        out.seq.append(nr + size_t(id) * L, tail ? L : offset[id]);
    });
}

std::vector<uint64_t> pack_ref(const std::string& s) {
    // compress.cu:219-246: ceil(len/32) words plus one zero pad word
    std::vector<uint64_t> b((s.size() + 31) / 32 + 1, 0);
    for (size_t i = 0; i < s.size(); ++i) b[i >> 5] |= uint64_t(enc(s[i])) << (62 - 2 * (i & 31));
    return b;
}

// ---------------------------------------------------------------- a9

namespace {
struct KmerIndex {
    uint32_t mask;
    std::vector<uint32_t> ranges, pos;
};

// compress.cu:362-409 in index order: bucket counts capped at 12, and each
// bucket keeps its first (lowest index) entries in descending slots.
void build_map_index(const uint64_t* ref, uint64_t start, uint64_t count, int k, int step, bool rc,
                     KmerIndex& ix) {
    uint32_t hs = hash_size_for(count);
    ix.mask = hs - 1;
    std::vector<uint8_t> cnt(size_t(hs) + 2, 0);
    std::vector<uint32_t> hv(count);
    for (uint64_t i = 0; i < count; ++i) {
        uint64_t km = word_unaligned(ref, start + i * step, k);
        if (rc) km = revcomp_kmer(km, k);
        hv[i] = uint32_t(murmur64(km) & ix.mask);
        if (cnt[hv[i]] < Params::bucket_limit) ++cnt[hv[i]];
    }
    ix.ranges.assign(size_t(hs) + 2, 0);
    uint32_t acc = 0;
    for (size_t h = 0; h < size_t(hs) + 2; ++h) { ix.ranges[h] = acc; acc += cnt[h]; }
    ix.pos.assign(acc + 2, 0);
    for (uint64_t i = 0; i < count; ++i) {
        uint32_t h = hv[i];
        if (cnt[h]) ix.pos[ix.ranges[h] + (--cnt[h])] = uint32_t(i);
    }
}
}  // namespace

void map_reads(const Params& p, const uint64_t* ref, size_t ref_len, const uint64_t* udb, size_t U,
               const char* ndb, size_t NN, MapResult& r, int threads) {
    // compress.cu:268-595 (init, index_and_mapping<false/true>, mapping)
    const int L = p.read_len, W = p.unit, k = Params::k1, step = Params::ref_step;
    const size_t total = U + NN;
    r.mm.assign(total, uint8_t(p.max_mismatch + 1));
    r.strand.assign(total, 0);
    r.pos.assign(total, 0);
    if (ref_len < size_t(k)) return;  // the reference cannot index a reference shorter than k
    const uint64_t index_count = (ref_len - k + 1 + step - 1) / step;
    std::vector<std::pair<uint64_t, uint64_t>> parts;
    if (index_count > (1ull << 30)) {
        uint64_t a = index_count / 2;
        parts = {{0, a}, {a * step, index_count - a}};
    } else {
        parts = {{0, index_count}};
    }
    for (int rc = 0; rc < 2; ++rc) {
        for (auto [start, count] : parts) {
            KmerIndex ix;
            build_map_index(ref, start, count, k, step, rc, ix);
#pragma omp parallel for schedule(dynamic, 256) num_threads(threads)
            for (size_t i = 0; i < total; ++i) {
                if (r.mm[i] <= Params::target_mm) continue;
                const bool isn = i >= U;
                const uint64_t* rd = isn ? nullptr : udb + i * W;
                const char* nd = isn ? ndb + (i - U) * L : nullptr;
                for (int j = 0; j + k <= L; j += Params::read_step) {
                    uint64_t key = isn ? kmer_from_ascii(nd + j, k) : word_at(rd, j, k);
                    uint32_t h = uint32_t(murmur64(key) & ix.mask);
                    uint32_t b = ix.ranges[h], e = ix.ranges[h + 1];
                    if (b == e) continue;
                    e = std::min(b + 12, e);
                    for (uint32_t q = b; q < e; ++q) {
                        uint64_t refpos = start + uint64_t(ix.pos[q]) * step;
                        uint64_t shift = rc ? uint64_t(L - k - j) : uint64_t(j);
                        if (refpos < shift) continue;
                        uint64_t mp = refpos - shift;
                        if (mp + L > ref_len) continue;
                        const int bound = r.mm[i];
                        int c = 0;
                        for (int o = 0; o < L && c < bound; ++o) {
                            int rb = code_at(ref, mp + o);
                            if (!isn) {
                                int qb = rc ? 3 - code_at(rd, L - 1 - o) : code_at(rd, o);
                                c += rb != qb;
                            } else {
                                char qc = rc ? comp_base(nd[L - 1 - o]) : nd[o];
                                c += "ACGT"[rb] != qc;
                            }
                        }
                        if (c < bound) {
                            r.strand[i] = uint8_t(rc);
                            r.pos[i] = mp;
                            r.mm[i] = uint8_t(c);
                            if (r.mm[i] <= Params::target_mm) goto next_read;
                        }
                    }
                }
            next_read:;
            }
        }
    }
}

// ---------------------------------------------------------------- a12

namespace {
constexpr int RM_K = 36, RM_SRC_STEP = 5, RM_DEST_STEP = 3, RM_MIN = 50, RM_BUCKET = 12;

// maRushPrime1Hash (compress.cu:597-631) over 36 symbols: nine
// little-endian 32-bit groups, each plus its group index, xor-multiplied.
template <class Sym>
uint32_t marush36(Sym sym) {
    uint64_t h = RM_K;
    for (uint32_t j = 0; j < RM_K / 4; ++j) {
        uint32_t v = uint32_t(uint8_t(sym(4 * j))) | uint32_t(uint8_t(sym(4 * j + 1))) << 8 |
                     uint32_t(uint8_t(sym(4 * j + 2))) << 16 | uint32_t(uint8_t(sym(4 * j + 3))) << 24;
        v += j;
        h ^= v;
        h *= 171717;
    }
    return uint32_t(h);
}

struct Match {
    uint64_t src, len, dst;
    bool operator<(const Match& o) const {
        if (dst != o.dst) return dst < o.dst;
        if (src != o.src) return src < o.src;
        return len < o.len;
    }
    bool operator==(const Match& o) const { return src == o.src && len == o.len && dst == o.dst; }
};
}  // namespace

void refmatch_index(const uint64_t* ref, uint64_t ref_len, RefMatcherIndex& ix) {
    // compress.cu:697-744
    ix.ref = ref;
    ix.ref_len = ref_len;
    if (ref_len < uint64_t(RM_K)) throw std::runtime_error("RefMatcher: reference shorter than 36");
    uint64_t count = (ref_len - RM_K + 1 + RM_SRC_STEP - 1) / RM_SRC_STEP;
    uint32_t hs = hash_size_for(count);
    ix.mask = hs - 1;
    std::vector<uint8_t> cnt(size_t(hs) + 2, 0);
    std::vector<uint32_t> hv(count);
    for (uint64_t i = 0; i < count; ++i) {
        uint64_t pos = i * RM_SRC_STEP;
        hv[i] = marush36([&](int t) { return base_at(ref, pos + t); }) & ix.mask;
        if (cnt[hv[i]] < RM_BUCKET) ++cnt[hv[i]];
    }
    ix.key_ranges.assign(size_t(hs) + 2, 0);
    uint32_t acc = 0;
    for (size_t h = 0; h < size_t(hs) + 2; ++h) { ix.key_ranges[h] = acc; acc += cnt[h]; }
    ix.pos_array.assign(acc + 2, 0);
    for (uint64_t i = 0; i < count; ++i)
        if (cnt[hv[i]]) ix.pos_array[ix.key_ranges[hv[i]] + (--cnt[hv[i]])] = uint32_t(i);
}

static void write_frugal(std::string& s, uint64_t v) {  // PgSAHelpers::writeUIntByteFrugal
    while (v >= 128) {
        s.push_back(char(128 + (v % 128)));
        v /= 128;
    }
    s.push_back(char(v));
}

void refmatch_apply(const RefMatcherIndex& ix, std::string& dest, bool dest_has_n, bool dest_is_ref,
                    std::string& map_off, std::string& map_len, int threads) {
    // compress.cu:746-992
    map_off.clear();
    map_len.clear();
    const uint64_t dl = dest.size(), rl = ix.ref_len;
    if (dl == 0) return;
    std::string rcd(dl, 'N');
    for (uint64_t i = 0; i < dl; ++i) rcd[i] = comp_base(dest[dl - 1 - i]);
    const uint64_t dic = dl >= uint64_t(RM_K) ? (dl - RM_K + 1 + RM_DEST_STEP - 1) / RM_DEST_STEP : 0;
    const uint64_t cap = uint64_t(double(dic) * (dest_is_ref ? 0.2 : 0.21));
    // the packed copy of the reverse-complemented dest has a zero pad; reads
    // past it see 'A' (code 0)
    std::vector<uint64_t> bin;
    if (!dest_has_n) bin = pack_ref(rcd);
    auto dsym = [&](uint64_t i) -> char {
        if (dest_has_n) return i < dl ? rcd[i] : '\0';
        return (i >> 5) < bin.size() ? base_at(bin.data(), i) : 'A';
    };
    auto dword = [&](uint64_t off) -> uint64_t {
        uint64_t v = 0;
        for (int t = 0; t < 32; ++t) v = (v << 2) | uint64_t(enc(dsym(off + t)));
        return v;
    };
    auto rsym = [&](uint64_t i) { return base_at(ix.ref, i); };
    std::vector<Match> m;
    auto probe = [&](uint64_t dpos, Match& found) -> bool {
        uint32_t h = marush36([&](int t) { return dsym(dpos + t); }) & ix.mask;
        uint64_t b = ix.key_ranges[h], e = ix.key_ranges[h + 1];
        for (uint64_t j = b; j < e; ++j) {
            uint64_t spos = uint64_t(ix.pos_array[j]) * RM_SRC_STEP;
            if (!dest_has_n && dest_is_ref && (dl - spos < dpos)) continue;
            uint64_t dc = dpos, sc = spos;
            uint64_t p1 = dc + RM_K - 1, p2 = sc + RM_K - 1;
            while (++p1 != dl && ++p2 != rl && dsym(p1) == rsym(p2)) {}
            uint64_t right = p1;
            p1 = dc;
            p2 = sc;
            while (p1 != 0 && p2 != 0 && dsym(--p1) == rsym(--p2)) {}
            if (right - p1 > uint64_t(RM_MIN)) {
                int cl;
                if (!dest_has_n) {
                    if (dword(dc) != word_unaligned(ix.ref, sc, 32)) continue;
                    dc += 32;
                    sc += 32;
                    cl = RM_K - 32;
                } else {
                    cl = RM_K;
                }
                while (cl && dsym(dc++) == rsym(sc++)) --cl;
                if (cl == 0) {
                    found = {p2 + 1, right - p1 - 1, p1 + 1};
                    return true;
                }
            }
        }
        return false;
    };
    // Probe groups are independent (the first hit of a group wins) and read
    // only the index and the strings, so they are searched in parallel and
    // their matches taken in group order.
    // Without N: groups of 4 probes; the probes of the last group at index
    // dic or later take no hit (their 36-mer runs past the end, and a hit
    // there would end past it, which the reference's compaction cannot
    // handle: compress.cu:910-913, 960-963).  With N: one probe per group.
    const uint64_t per = dest_has_n ? 1 : 4;
    const uint64_t groups = (dic + per - 1) / per;
    std::vector<Match> found(groups);
    std::vector<uint8_t> hit(groups, 0);
#pragma omp parallel for schedule(dynamic, 256) num_threads(threads)
    for (uint64_t i = 0; i < groups; ++i)
        for (uint64_t q = 0; q < per && i * per + q < dic; ++q)
            if (probe((i * per + q) * RM_DEST_STEP, found[i])) {
                hit[i] = 1;
                break;
            }
    for (uint64_t i = 0; i < groups; ++i)
        if (hit[i]) m.push_back(found[i]);
    if (m.size() > cap) m.resize(cap);  // capacity drop, first entries in index order kept
    if (m.empty()) return;
    for (auto& x : m) x.dst = dl - (x.dst + x.len);
    if (dest_is_ref) {
        for (auto& x : m) {
            if (x.src > x.dst) std::swap(x.src, x.dst);
            uint64_t end = x.src + x.len;
            if (end > x.dst) {
                uint64_t margin = (end - x.dst + 1) / 2;
                x.len -= margin;
                x.dst += margin;
            }
        }
    }
    std::sort(m.begin(), m.end());
    m.erase(std::unique(m.begin(), m.end()), m.end());
    write_frugal(map_len, RM_MIN);
    const bool std32 = rl <= 0xFFFFFFFFull;
    uint64_t pos = 0, npos = 0;
    for (auto& x : m) {
        if (x.dst < pos) {
            uint64_t ov = pos - x.dst;
            if (ov >= x.len) continue;
            x.len -= ov;
            x.dst += ov;
        }
        if (x.len < uint64_t(RM_MIN)) continue;
        uint64_t n = x.dst - pos;
        std::memmove(&dest[npos], &dest[pos], n);
        npos += n;
        dest[npos++] = '%';
        if (std32) {
            uint32_t v = uint32_t(x.src);
            map_off.append(reinterpret_cast<const char*>(&v), 4);
        } else {
            map_off.append(reinterpret_cast<const char*>(&x.src), 8);
        }
        write_frugal(map_len, x.len - RM_MIN);
        pos = x.dst + x.len;
    }
    uint64_t n = dl - pos;
    std::memmove(&dest[npos], &dest[pos], n);
    npos += n;
    dest.resize(npos);
}

}  // namespace oracle
