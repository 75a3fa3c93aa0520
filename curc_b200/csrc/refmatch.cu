// a12: reverse-complement repeat removal in the pseudogenomes.
//
// Reference: RefMatcher compress.cu:631-1001.  An index of 36-mers of the
// main pseudogenome every 5 bases (maRushPrime1 hash, buckets capped at 12);
// each destination string is reverse complemented and probed every 3 bases
// (in segments of 4 probes for packed destinations, the first hit ending the
// segment); a hit is extended both ways and kept when the extension spans
// more than 50 bases and the whole 36-mer matches.  Hits become (src, len,
// dst) triples that are sorted, deduplicated and applied: each kept span of
// the destination is replaced by '%', its source offset goes to MapOff and
// its length to MapLen.
//
// Canonical semantics: the reference appends hits with atomicAdd and drops
// those beyond its capacity in arrival order; here the hits kept are the
// first `capacity` in probe order.  The index buckets hold the first 12
// positions (as in mapper.cu).
//
// B200 design: one thread per probe, the four probes of a segment in
// adjacent lanes; the 36-mer is compared before the match is extended, and
// a maximal match met by a run of consecutive segments is extended once; the
// extensions compare 32 bases per step with XOR and count-leading-zeros
// instead of one base per step; the triples are ordered with three stable
// radix passes; the acceptance walk (each decision depends on the end of the
// previous kept span) is rewritten as a successor chain followed by binary
// lifting; the map streams and the string compaction are built in parallel
// from scans over the kept spans.
#include <cstring>

#include "block.cuh"

namespace curc {

namespace {

constexpr int RM_K = 36, RM_SRC_STEP = 5, RM_DEST_STEP = 3, RM_MIN = 50;

struct Hit {
    uint64_t src, len, dst;
};

// The four bases of one byte of a packed word (first base in the top two
// bits) as ASCII bytes, first base lowest: byte c of 'A','C','G','T' for each
// code, selected with one byte permute.
__device__ __forceinline__ uint32_t ascii4(uint32_t b) {
    const uint32_t sel = (b >> 6) | ((b >> 4) & 3u) << 4 | ((b >> 2) & 3u) << 8 | (b & 3u) << 12;
    return __byte_perm(0x54474341u, 0u, sel);
}

// maRushPrime1HashBinary<36> (compress.cu:597-615): the 36 bases as nine
// little-endian words of four ASCII characters, each plus its index, folded
// by xor and multiply.
__device__ __forceinline__ uint32_t marush_packed(const uint64_t* bits, uint64_t pos) {
    const uint64_t x = word_unaligned(bits, pos, 32);
    const uint32_t t = uint32_t(word_unaligned(bits, pos + 32, 4));
    uint64_t h = RM_K;
#pragma unroll
    for (uint32_t j = 0; j < 8; ++j) {
        h ^= ascii4(uint32_t(x >> (56 - 8 * j)) & 0xFFu) + j;
        h *= 171717;
    }
    h ^= ascii4(t) + 8u;
    h *= 171717;
    return uint32_t(h);
}

// maRushPrime1HashChar<36> (compress.cu:617-629)
__device__ __forceinline__ uint32_t marush_ascii(const uint8_t* s) {
    uint64_t h = RM_K;
#pragma unroll
    for (uint32_t j = 0; j < RM_K / 4; ++j) {
        uint32_t v = uint32_t(s[4 * j]) | uint32_t(s[4 * j + 1]) << 8 | uint32_t(s[4 * j + 2]) << 16 |
                     uint32_t(s[4 * j + 3]) << 24;
        v += j;
        h ^= v;
        h *= 171717;
    }
    return uint32_t(h);
}

__global__ void rm_hash_kernel(const uint64_t* __restrict__ ref, uint64_t count, uint32_t mask,
                               uint32_t* __restrict__ hv, uint32_t* __restrict__ idx) {
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += uint64_t(gridDim.x) * blockDim.x) {
        hv[i] = marush_packed(ref, i * RM_SRC_STEP) & mask;
        idx[i] = uint32_t(i);
    }
}

// reverse complement of an ASCII string
__global__ void rc_ascii_kernel(const uint8_t* __restrict__ in, uint64_t n, uint8_t* __restrict__ out) {
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
        out[i] = uint8_t(comp_char(char(in[n - 1 - i])));
}

struct RmIndex {
    const uint64_t* ref;
    uint64_t rl;
    uint32_t mask;
    const uint32_t* kr;
    const uint32_t* pos;
};

// Number of equal bases of a[ao..) and b[bo..) going right, at most lim.
__device__ __forceinline__ uint64_t match_right(const uint64_t* a, uint64_t ao, const uint64_t* b, uint64_t bo,
                                                uint64_t lim) {
    uint64_t k = 0;
    while (k < lim) {
        const int nb = lim - k < 32 ? int(lim - k) : 32;
        const uint64_t x = word_unaligned(a, ao + k, nb) ^ word_unaligned(b, bo + k, nb);
        if (x) return k + (__clzll(x) - (64 - 2 * nb)) / 2;
        k += nb;
    }
    return lim;
}

// Number of equal bases of a[..ao) and b[..bo) going left, at most lim.
__device__ __forceinline__ uint64_t match_left(const uint64_t* a, uint64_t ao, const uint64_t* b, uint64_t bo,
                                               uint64_t lim) {
    uint64_t k = 0;
    while (k < lim) {
        const int nb = lim - k < 32 ? int(lim - k) : 32;
        const uint64_t x = word_unaligned(a, ao - k - nb, nb) ^ word_unaligned(b, bo - k - nb, nb);
        if (x) return k + uint64_t(__ffsll(x) - 1) / 2;  // equal 2-bit groups from the right
        k += nb;
    }
    return lim;
}

// Packed destination (reverse complemented, dl bases, zero padded): the
// reference's probe of one destination position against one bucket
// (compress.cu:758-802).  A bucket entry is taken when the match through it
// spans more than 50 bases and its whole 36-mer is equal; both tests are
// required, so the 36-mer is compared first, and the span test needs at most
// 15 bases of extension on each side (36 + right + left + 1 > 50).  Returns
// the source position of the first entry taken.
__device__ bool probe_candidate(const RmIndex& ix, const uint64_t* dest, uint64_t dl, uint64_t dpad, uint64_t dpos,
                                bool dest_is_ref, uint64_t* spos_out) {
    const uint32_t h = marush_packed(dest, dpos) & ix.mask;
    const uint32_t b = ix.kr[h], e = ix.kr[h + 1];
    if (b == e) return false;
    const uint64_t k32 = word_unaligned(dest, dpos, 32), k4 = word_unaligned(dest, dpos + 32, 4);
    const uint64_t d0 = dpos + RM_K;
    const uint64_t dlim = d0 <= dl ? dl - d0 : dpad - d0;  // bases readable on the dest side
    for (uint32_t j = b; j < e; ++j) {
        const uint64_t spos = uint64_t(ix.pos[j]) * RM_SRC_STEP;
        if (dest_is_ref && (dl - spos < dpos)) continue;
        if (word_unaligned(ix.ref, spos, 32) != k32 || word_unaligned(ix.ref, spos + 32, 4) != k4) continue;
        const uint64_t s0 = spos + RM_K;
        const uint64_t slim = s0 <= ix.rl ? ix.rl - s0 : 0;
        const uint64_t run = match_right(dest, d0, ix.ref, s0, min(min(dlim, slim), uint64_t(15)));
        const uint64_t lmax = min(dpos, spos);
        const uint64_t k = match_left(dest, dpos, ix.ref, spos, min(lmax, uint64_t(15)));
        if (run + k + (k < lmax ? 1 : 0) + RM_K > uint64_t(RM_MIN)) {
            *spos_out = spos;
            return true;
        }
    }
    return false;
}

// The maximal match through an accepted probe: extended right from the end
// of the 36-mer and left from its start, as the reference does.
__device__ Hit extend_full(const RmIndex& ix, const uint64_t* dest, uint64_t dl, uint64_t dpad, uint64_t dpos,
                           uint64_t spos) {
    const uint64_t d0 = dpos + RM_K, s0 = spos + RM_K;
    const uint64_t dlim = d0 <= dl ? dl - d0 : dpad - d0;
    const uint64_t slim = s0 <= ix.rl ? ix.rl - s0 : 0;
    const uint64_t right = d0 + match_right(dest, d0, ix.ref, s0, min(dlim, slim));
    const uint64_t lmax = min(dpos, spos);
    const uint64_t k = match_left(dest, dpos, ix.ref, spos, lmax);
    const uint64_t p1 = k < lmax ? dpos - 1 - k : dpos - k;
    const uint64_t p2 = k < lmax ? spos - 1 - k : spos - k;
    return Hit{p2 + 1, right - p1 - 1, p1 + 1};
}

// One thread per probe; the four probes of a segment sit in four adjacent
// lanes and the segment takes its first accepting probe (the reference's
// segment stops at its first hit, compress.cu:746-807).  cand[seg] = (dest, source) position.
// Probes at index dic or later (the tail of the last segment) take no hit:
// their 36-mer runs past the destination end, and in the reference any hit
// there ends past it too, so its length arithmetic (compress.cu:910-913)
// wraps and its compaction (compress.cu:960-963) moves out of bounds.
__global__ void __launch_bounds__(256) probe_segments_kernel(RmIndex ix, const uint64_t* __restrict__ dest, uint64_t dl,
                                                             uint64_t dpad, uint64_t segs, uint64_t dic,
                                                             bool dest_is_ref, uint8_t* __restrict__ flag,
                                                             ulonglong2* __restrict__ cand) {
    const uint64_t P = segs * 4;
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    // lanes of a warp share i - lane, so the warp stays converged for the ballot
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i - lane < P; i += stride) {
        uint64_t sp = 0;
        const bool hit = i < dic && probe_candidate(ix, dest, dl, dpad, i * RM_DEST_STEP, dest_is_ref, &sp);
        const uint32_t g = (__ballot_sync(0xFFFFFFFFu, hit) >> (lane & ~3u)) & 0xFu;
        if (i < P) {
            if ((lane & 3u) == 0) flag[i >> 2] = g != 0;
            if (g && (lane & 3u) == uint32_t(__ffs(g) - 1)) cand[i >> 2] = make_ulonglong2(i * RM_DEST_STEP, sp);
        }
    }
}

// Segment j lies in the same maximal match as segment j-1: both accepted a
// probe on the same diagonal (source - dest), and their 36-mers, at most 21
// bases apart, overlap, so extending either gives the same span (both right
// limits are the destination end).
__device__ __forceinline__ bool rm_follows(const uint8_t* flag, const ulonglong2* cand, uint64_t j, uint64_t dl) {
    if (j == 0 || !flag[j - 1]) return false;
    const ulonglong2 c = cand[j], p = cand[j - 1];
    return c.x + RM_K <= dl && c.y - c.x == p.y - p.x;
}

// The first segment of each run extends its match once and writes the hit
// for the whole run.
__global__ void extend_runs_kernel(RmIndex ix, const uint64_t* __restrict__ dest, uint64_t dl, uint64_t dpad,
                                   uint64_t segs, const uint8_t* __restrict__ flag,
                                   const ulonglong2* __restrict__ cand, Hit* __restrict__ hits) {
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < segs; i += uint64_t(gridDim.x) * blockDim.x) {
        if (!flag[i] || rm_follows(flag, cand, i, dl)) continue;
        const Hit h = extend_full(ix, dest, dl, dpad, cand[i].x, cand[i].y);
        hits[i] = h;
        for (uint64_t j = i + 1; j < segs && flag[j] && rm_follows(flag, cand, j, dl); ++j) hits[j] = h;
    }
}

__global__ void probe_ascii_kernel(RmIndex ix, const uint8_t* __restrict__ dest, uint64_t dl, uint64_t dic,
                                   uint8_t* __restrict__ flag, Hit* __restrict__ hits) {
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < dic; i += uint64_t(gridDim.x) * blockDim.x) {
        const uint64_t dpos = i * RM_DEST_STEP;
        const uint32_t h = marush_ascii(dest + dpos) & ix.mask;
        const uint32_t b = ix.kr[h], e = ix.kr[h + 1];
        uint8_t f = 0;
        for (uint32_t j = b; j < e; ++j) {
            const uint64_t spos = uint64_t(ix.pos[j]) * RM_SRC_STEP;
            uint64_t p1 = dpos + RM_K - 1, p2 = spos + RM_K - 1;
            while (++p1 != dl && ++p2 != ix.rl && dest[p1] == uint8_t("ACGT"[code_at(ix.ref, p2)])) {}
            const uint64_t right = p1;
            p1 = dpos;
            p2 = spos;
            while (p1 != 0 && p2 != 0 && dest[--p1] == uint8_t("ACGT"[code_at(ix.ref, --p2)])) {}
            if (right - p1 > uint64_t(RM_MIN)) {
                int cl = RM_K;
                uint64_t dc = dpos, sc = spos;
                while (cl && dest[dc++] == uint8_t("ACGT"[code_at(ix.ref, sc++)])) --cl;
                if (cl == 0) {
                    hits[i] = Hit{p2 + 1, right - p1 - 1, p1 + 1};
                    f = 1;
                    break;
                }
            }
        }
        flag[i] = f;
    }
}

__global__ void gather_hits_kernel(const Hit* __restrict__ in, const uint32_t* __restrict__ sel, uint32_t c,
                                   uint64_t dl, bool dest_is_ref, Hit* __restrict__ out) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= c) return;
    Hit h = in[sel[t]];
    h.dst = dl - (h.dst + h.len);  // back to forward coordinates (compress.cu:903-908)
    if (dest_is_ref) {             // compress.cu:910-927
        if (h.src > h.dst) {
            const uint64_t x = h.src;
            h.src = h.dst;
            h.dst = x;
        }
        const uint64_t end = h.src + h.len;
        if (end > h.dst) {
            const uint64_t margin = (end - h.dst + 1) / 2;
            h.len -= margin;
            h.dst += margin;
        }
    }
    out[t] = h;
}

__global__ void hit_key_kernel(const Hit* __restrict__ h, const uint32_t* __restrict__ idx, uint32_t c, int field,
                               uint64_t* __restrict__ key) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= c) return;
    const Hit x = h[idx[t]];
    key[t] = field == 0 ? x.len : (field == 1 ? x.src : x.dst);
}

__global__ void hit_unique_kernel(const Hit* __restrict__ h, const uint32_t* __restrict__ idx, uint32_t c,
                                  uint8_t* __restrict__ keep, Hit* __restrict__ sorted) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= c) return;
    const Hit x = h[idx[t]];
    sorted[t] = x;
    bool k = true;
    if (t > 0) {
        const Hit y = h[idx[t - 1]];
        k = !(x.src == y.src && x.len == y.len && x.dst == y.dst);
    }
    keep[t] = k;
}

__global__ void compact_hits_kernel(const Hit* __restrict__ in, const uint32_t* __restrict__ sel, uint32_t c,
                                    Hit* __restrict__ out) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < c) out[t] = in[sel[t]];
}

// compress.cu:946-992, the acceptance walk over the sorted distinct hits:
// a hit starting before the end `pos` of the last kept span is trimmed to
// start there (or dropped when covered), and kept when 50 or more bases
// remain; a kept hit sets pos to its end.  Trimming keeps the end, so with
// end_i = dst_i + len_i, hit i is kept iff len_i >= 50 and end_i >= pos + 50,
// and then pos = end_i.  The kept hits are therefore the chain
//   start -> nxt(start) -> nxt(nxt(start)) -> ...
// where nxt(j) is the first i > j with len_i >= 50 and end_i >= end_j + 50
// (the start has end 0).  nxt is found for every hit at once by descending
// a sparse table of range maxima of the eligible ends, and the chain is
// followed by binary lifting, so no step is sequential.  Node c is the
// start and c + 1 the end of the chain.

// eligible ends: level 0 of the range-maximum table
__global__ void accept_ends_kernel(const Hit* __restrict__ h, uint32_t c, uint64_t* __restrict__ m0) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < c) m0[i] = h[i].len >= uint64_t(RM_MIN) ? h[i].dst + h[i].len : 0;
}

// level k from level k-1: maxima of [i, i + 2^k), valid where i + 2^k <= c
__global__ void range_max_kernel(const uint64_t* __restrict__ prev, uint32_t c, uint32_t half,
                                 uint64_t* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < c) out[i] = i + half < c ? max(prev[i], prev[i + half]) : prev[i];
}

__global__ void accept_next_kernel(const Hit* __restrict__ h, const uint64_t* __restrict__ M, uint32_t c, int levels,
                                   uint32_t* __restrict__ J0) {
    const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u > c + 1) return;
    if (u == c + 1) {
        J0[u] = c + 1;
        return;
    }
    uint32_t p;
    uint64_t T;
    if (u == c) {
        p = 0;
        T = RM_MIN;
    } else if (h[u].len < uint64_t(RM_MIN)) {
        J0[u] = c + 1;  // never kept, never followed
        return;
    } else {
        p = u + 1;
        T = h[u].dst + h[u].len + RM_MIN;
    }
    // skip the longest run of ends below T: its length bit by bit
    for (int k = levels - 1; k >= 0; --k)
        if (uint64_t(p) + (1ull << k) <= c && M[uint64_t(k) * c + p] < T) p += 1u << k;
    J0[u] = p < c ? p : c + 1;
}

__global__ void lift_square_kernel(const uint32_t* __restrict__ Jk, uint32_t nodes, uint32_t* __restrict__ Jn) {
    const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u < nodes) Jn[u] = Jk[Jk[u]];
}

__device__ __forceinline__ uint32_t lift(const uint32_t* J, uint32_t nodes, uint32_t u, uint32_t t) {
    for (int k = 0; t; ++k, t >>= 1)
        if (t & 1u) u = J[uint64_t(k) * nodes + u];
    return u;
}

// The t-th kept hit (t >= 1) and its trimmed start.
__global__ void accept_chain_kernel(const Hit* __restrict__ h, uint32_t c, const uint32_t* __restrict__ J,
                                    uint8_t* __restrict__ kept, uint64_t* __restrict__ adst,
                                    uint64_t* __restrict__ alen) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (t > c) return;
    const uint32_t nodes = c + 2;
    const uint32_t i = lift(J, nodes, c, t);
    if (i >= c) return;  // the chain is shorter than t
    const uint32_t pr = lift(J, nodes, c, t - 1);
    const uint64_t pos = pr == c ? 0 : h[pr].dst + h[pr].len;
    const uint64_t end = h[i].dst + h[i].len;
    const uint64_t d = max(h[i].dst, pos);
    kept[i] = 1;
    adst[i] = d;
    alen[i] = end - d;
}

__device__ __forceinline__ uint32_t frugal_size(uint64_t v) {
    uint32_t n = 1;
    while (v >= 128) {
        v /= 128;
        ++n;
    }
    return n;
}

// Per kept span k (hit i = sel[k]): span bounds, removed length, MapOff
// entry, and the size of its MapLen entry.
__global__ void kept_spans_kernel(const uint32_t* __restrict__ sel, uint32_t K, const Hit* __restrict__ h,
                                  const uint64_t* __restrict__ adst, const uint64_t* __restrict__ alen, bool std32,
                                  uint64_t* __restrict__ sd, uint64_t* __restrict__ se, uint64_t* __restrict__ rm,
                                  uint32_t* __restrict__ lsize, uint8_t* __restrict__ map_off) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= K) return;
    const uint32_t i = sel[k];
    const uint64_t d = adst[i], l = alen[i];
    sd[k] = d;
    se[k] = d + l;
    rm[k] = l - 1;
    lsize[k] = frugal_size(l - RM_MIN);
    const uint64_t src = h[i].src;
    if (std32) {
        const uint32_t v = uint32_t(src);
        for (int t = 0; t < 4; ++t) map_off[uint64_t(k) * 4 + t] = uint8_t(v >> (8 * t));
    } else {
        for (int t = 0; t < 8; ++t) map_off[uint64_t(k) * 8 + t] = uint8_t(src >> (8 * t));
    }
}

// MapLen: LEB128(50) then LEB128(len - 50) per kept span.
__global__ void map_len_kernel(const uint32_t* __restrict__ sel, uint32_t K, const uint64_t* __restrict__ alen,
                               const uint32_t* __restrict__ loff, uint8_t* __restrict__ map_len) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k == 0) map_len[0] = uint8_t(RM_MIN);
    if (k >= K) return;
    uint64_t v = alen[sel[k]] - RM_MIN;
    uint64_t o = 1 + uint64_t(loff[k]);
    while (v >= 128) {
        map_len[o++] = uint8_t(128 + (v % 128));
        v /= 128;
    }
    map_len[o] = uint8_t(v);
}

// Each kept span [sd_k, se_k) becomes one '%'; every other symbol moves left
// by the symbols removed before it.
__global__ void compact_string_kernel(const uint8_t* __restrict__ in, uint64_t dl, const uint64_t* __restrict__ sd,
                                      const uint64_t* __restrict__ se, const uint64_t* __restrict__ removed,
                                      uint64_t kept, uint8_t* __restrict__ out) {
    for (uint64_t q = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < dl; q += uint64_t(gridDim.x) * blockDim.x) {
        uint64_t lo = 0, cnt = kept;  // lo = number of spans starting at or before q
        while (cnt > 0) {
            const uint64_t step = cnt / 2, it = lo + step;
            if (sd[it] <= q) {
                lo = it + 1;
                cnt -= step + 1;
            } else {
                cnt = step;
            }
        }
        if (lo > 0 && q < se[lo - 1]) {
            if (q == sd[lo - 1]) out[q - removed[lo - 1]] = '%';
            continue;
        }
        out[q - removed[lo]] = in[q];
    }
}

__global__ void rm_bucket_caps_kernel(const uint32_t* __restrict__ hv, uint64_t count, uint32_t* __restrict__ cnt) {
    for (uint64_t j = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < count; j += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t h = hv[j];
        if (j > 0 && hv[j - 1] == h) continue;
        uint32_t c = 1;
        while (c < 12 && j + c < count && hv[j + c] == h) ++c;
        cnt[h] = c;
    }
}

__global__ void rm_bucket_fill_kernel(const uint32_t* __restrict__ hv, const uint32_t* __restrict__ idx,
                                      uint64_t count, const uint32_t* __restrict__ kr, uint32_t* __restrict__ pos) {
    for (uint64_t j = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < count; j += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t h = hv[j];
        uint32_t rank = 0;
        while (rank < 12 && rank < j && hv[j - 1 - rank] == h) ++rank;
        const uint32_t b = kr[h], c = kr[h + 1] - b;
        if (rank < c) pos[b + c - 1 - rank] = idx[j];
    }
}

inline int log2_ceil(uint32_t x) {
    int b = 0;
    while ((1u << b) < x) ++b;
    return b;
}

// Device views of one destination's results (valid until the arena region
// is reused: the caller copies them out before the next destination).
struct RmResult {
    const uint8_t* seq = nullptr;
    uint64_t seq_len = 0;
    const uint8_t* map_off = nullptr;
    uint64_t off_len = 0;
    const uint8_t* map_len = nullptr;
    uint64_t len_len = 0;
};

// One destination (compress.cu:856-993).  `dest` is the ASCII string on the
// device (forward strand).
void refmatch_one(const RmIndex& ix, const uint8_t* dest, uint64_t dl, bool has_n, bool dest_is_ref, RmResult& r,
                  Arena& a, cudaStream_t s) {
    r = RmResult{};
    r.seq = dest;  // unchanged unless spans are kept
    r.seq_len = dl;
    const uint64_t dic = dl >= uint64_t(RM_K) ? (dl - RM_K + 1 + RM_DEST_STEP - 1) / RM_DEST_STEP : 0;
    const uint64_t cap = uint64_t(double(dic) * (dest_is_ref ? 0.2 : 0.21));
    if (dic == 0 || ix.rl < uint64_t(RM_K)) return;
    auto mk = a.mark();
    SubStage sp_probe(dest_is_ref ? "refmatch.probe_self" : "refmatch.probe_unmapped");
    uint8_t* rc = a.alloc<uint8_t>(dl + 64);
    rc_ascii_kernel<<<grid_for(dl, 256, 8), 256, 0, s>>>(dest, dl, rc);
    CURC_LAUNCH_CHECK();
    const uint64_t nslots = has_n ? dic : div_up(dic, 4);
    uint8_t* flag = a.alloc<uint8_t>(nslots);
    Hit* hits = a.alloc<Hit>(nslots);
    if (!has_n) {
        const uint64_t words = (dl + 31) / 32 + 8;
        uint64_t* packed = a.alloc<uint64_t>(words);
        CURC_CHECK(cudaMemsetAsync(packed, 0, words * 8, s));
        pack_ascii_ref(rc, dl, packed, s);
        const uint64_t dpad = (words - 1) * 32;
        ulonglong2* cand = a.alloc<ulonglong2>(nslots);
        probe_segments_kernel<<<resident_grid(probe_segments_kernel, 256, nslots * 4), 256, 0, s>>>(
            ix, packed, dl, dpad, nslots, dic, dest_is_ref, flag, cand);
        CURC_LAUNCH_CHECK();
        extend_runs_kernel<<<grid_for(nslots, 256), 256, 0, s>>>(ix, packed, dl, dpad, nslots, flag, cand, hits);
    } else {
        CURC_CHECK(cudaMemsetAsync(rc + dl, 0, 64, s));
        probe_ascii_kernel<<<grid_for(nslots, 128), 128, 0, s>>>(ix, rc, dl, dic, flag, hits);
    }
    CURC_LAUNCH_CHECK();
    uint32_t* cnt = a.alloc<uint32_t>(4);
    uint32_t* sel = a.alloc<uint32_t>(nslots);
    select_indices(flag, sel, nslots, cnt, a, s);
    uint32_t c = read_scalar(cnt, s);
    sp_probe.stop();
    if (c > cap) c = uint32_t(cap);  // capacity: the first hits in probe order
    if (c == 0) {
        a.release(mk);
        return;
    }
    SubStage sp_sort("refmatch.sort_unique");
    Hit* hv = a.alloc<Hit>(c);
    gather_hits_kernel<<<grid_for(c, 256), 256, 0, s>>>(hits, sel, c, dl, dest_is_ref, hv);
    CURC_LAUNCH_CHECK();
    // sort by (dst, src, len): three stable passes, least significant first
    uint32_t* idx = a.alloc<uint32_t>(c);
    uint64_t* key = a.alloc<uint64_t>(c);
    iota(idx, c, s);
    for (int field = 0; field < 3; ++field) {
        hit_key_kernel<<<grid_for(c, 256), 256, 0, s>>>(hv, idx, c, field, key);
        CURC_LAUNCH_CHECK();
        radix_sort_pairs<uint64_t, uint32_t>(key, idx, c, 0, 64, a, s);
    }
    uint8_t* keepf = a.alloc<uint8_t>(c);
    Hit* sorted = a.alloc<Hit>(c);
    hit_unique_kernel<<<grid_for(c, 256), 256, 0, s>>>(hv, idx, c, keepf, sorted);
    CURC_LAUNCH_CHECK();
    uint32_t* sel2 = a.alloc<uint32_t>(c);
    select_indices(keepf, sel2, c, cnt + 1, a, s);
    const uint32_t cu = read_scalar(cnt + 1, s);
    Hit* uniq = a.alloc<Hit>(cu);
    compact_hits_kernel<<<grid_for(cu, 256), 256, 0, s>>>(sorted, sel2, cu, uniq);
    CURC_LAUNCH_CHECK();
    sp_sort.stop();
    SubStage sp_accept("refmatch.accept");
    uint8_t* keptf = a.alloc<uint8_t>(cu);
    uint64_t* adst = a.alloc<uint64_t>(cu);
    uint64_t* alen = a.alloc<uint64_t>(cu);
    {
        int levels = 1;  // range-maximum levels: 2^(levels-1) <= cu
        while ((2ull << (levels - 1)) <= cu) ++levels;
        int lifts = 1;   // lifting levels: 2^lifts > cu
        while ((1ull << lifts) <= cu) ++lifts;
        const uint32_t nodes = cu + 2;
        uint64_t* M = a.alloc<uint64_t>(uint64_t(levels) * cu);
        uint32_t* J = a.alloc<uint32_t>(uint64_t(lifts) * nodes);
        const int gc = grid_for(cu, 256), gn = grid_for(nodes, 256);
        accept_ends_kernel<<<gc, 256, 0, s>>>(uniq, cu, M);
        CURC_LAUNCH_CHECK();
        for (int k = 1; k < levels; ++k) {
            range_max_kernel<<<gc, 256, 0, s>>>(M + uint64_t(k - 1) * cu, cu, 1u << (k - 1), M + uint64_t(k) * cu);
            CURC_LAUNCH_CHECK();
        }
        accept_next_kernel<<<gn, 256, 0, s>>>(uniq, M, cu, levels, J);
        CURC_LAUNCH_CHECK();
        for (int k = 1; k < lifts; ++k) {
            lift_square_kernel<<<gn, 256, 0, s>>>(J + uint64_t(k - 1) * nodes, nodes, J + uint64_t(k) * nodes);
            CURC_LAUNCH_CHECK();
        }
        CURC_CHECK(cudaMemsetAsync(keptf, 0, cu, s));
        accept_chain_kernel<<<gc, 256, 0, s>>>(uniq, cu, J, keptf, adst, alen);
        CURC_LAUNCH_CHECK();
    }
    uint32_t* ksel = a.alloc<uint32_t>(cu);
    select_indices(keptf, ksel, cu, cnt + 2, a, s);
    const uint32_t K = read_scalar(cnt + 2, s);
    const bool std32 = ix.rl <= 0xFFFFFFFFull;
    uint64_t* sd = a.alloc<uint64_t>(K + 1);
    uint64_t* se = a.alloc<uint64_t>(K + 1);
    uint64_t* removed = a.alloc<uint64_t>(K + 2);
    uint32_t* lsize = a.alloc<uint32_t>(K + 1);
    uint8_t* moff = a.alloc<uint8_t>(uint64_t(K) * 8 + 8);
    uint8_t* mlen = a.alloc<uint8_t>(uint64_t(K) * 10 + 16);
    if (K) {
        kept_spans_kernel<<<grid_for(K, 256), 256, 0, s>>>(ksel, K, uniq, adst, alen, std32, sd, se, removed, lsize,
                                                            moff);
        CURC_LAUNCH_CHECK();
    }
    exclusive_scan<uint64_t>(removed, removed, K, removed + K, a, s);
    exclusive_scan<uint32_t>(lsize, lsize, K, cnt + 3, a, s);
    map_len_kernel<<<grid_for(K ? K : 1, 256), 256, 0, s>>>(ksel, K, alen, lsize, mlen);
    CURC_LAUNCH_CHECK();
    uint64_t total_removed = 0;
    uint32_t len_bytes = 0;
    read_small(&total_removed, removed + K, 8, s);
    read_small(&len_bytes, cnt + 3, 4, s);
    uint64_t hi[4] = {K, uint64_t(K) * (std32 ? 4 : 8), 1 + uint64_t(len_bytes), dl - total_removed};
    r.map_off = moff;
    r.off_len = hi[1];
    r.map_len = mlen;
    r.len_len = hi[2];
    uint8_t* out = a.alloc<uint8_t>(hi[3] + 1);
    compact_string_kernel<<<grid_for(dl, 256, 8), 256, 0, s>>>(dest, dl, sd, se, removed, hi[0], out);
    CURC_LAUNCH_CHECK();
    r.seq = out;
    r.seq_len = hi[3];
    sp_accept.stop();
    a.release(mk);
}

}  // namespace

void Block::refmatch_all() {
    // compress.cu:2053-2069: index on the main pseudogenome, applied to the
    // unmapped, the unmapped-N and then the main pseudogenome itself.
    cudaStream_t s = stream;
    RmResult r;
    auto mk = arena.mark();
    RmIndex ix{hq.packed, hq.len, 0, nullptr, nullptr};
    const bool usable = hq.len >= uint64_t(RM_K);
    if (usable) {
        SubStage sub("refmatch.index");
        const uint64_t count = (hq.len - RM_K + 1 + RM_SRC_STEP - 1) / RM_SRC_STEP;
        if (count > (1ull << 30)) throw std::runtime_error("RefMatcher: pseudogenome above the 2^30-entry index");
        const uint32_t hs = hash_size_for(count);
        ix.mask = hs - 1;
        uint32_t* hv = arena.alloc<uint32_t>(count);
        uint32_t* idx = arena.alloc<uint32_t>(count);
        rm_hash_kernel<<<grid_for(count, 256, 4), 256, 0, s>>>(hq.packed, count, ix.mask, hv, idx);
        CURC_LAUNCH_CHECK();
        radix_sort_pairs<uint32_t, uint32_t>(hv, idx, count, 0, log2_ceil(hs), arena, s);
        uint32_t* kr = arena.alloc<uint32_t>(size_t(hs) + 2);
        CURC_CHECK(cudaMemsetAsync(kr, 0, (size_t(hs) + 2) * 4, s));
        rm_bucket_caps_kernel<<<grid_for(count, 256, 4), 256, 0, s>>>(hv, count, kr);
        CURC_LAUNCH_CHECK();
        exclusive_scan<uint32_t>(kr, kr, size_t(hs) + 2, nullptr, arena, s);
        uint32_t* pos = arena.alloc<uint32_t>(std::min<uint64_t>(count, uint64_t(hs) * 12) + 2);
        rm_bucket_fill_kernel<<<grid_for(count, 256, 4), 256, 0, s>>>(hv, idx, count, kr, pos);
        CURC_LAUNCH_CHECK();
        ix.kr = kr;
        ix.pos = pos;
    } else {
        ix.rl = 0;  // no index: every pseudogenome is kept as assembled
    }
    // results are copied out right after each destination, before the next
    // one reuses the scratch region
    refmatch_one(ix, lq.seq, lq.len, false, false, r, arena, s);
    keep("unmap_ref", r.seq, r.seq_len);
    keep("unmap_ref_off", r.map_off, r.off_len);
    keep("unmap_ref_len", r.map_len, r.len_len);
    const uint64_t un_len = r.seq_len;
    refmatch_one(ix, lqn.seq, lqn.len, true, false, r, arena, s);
    keep("unmap_n_ref", r.seq, r.seq_len);
    keep("unmap_n_ref_off", r.map_off, r.off_len);
    keep("unmap_n_ref_len", r.map_len, r.len_len);
    const uint64_t unn_len = r.seq_len;
    refmatch_one(ix, hq.seq, hq.len, false, true, r, arena, s);
    keep("ref", r.seq, r.seq_len);
    keep("ref_off", r.map_off, r.off_len);
    keep("ref_len_map", r.map_len, r.len_len);
    const uint64_t main_len = r.seq_len;
    arena.release(mk);
    const uint64_t sizes[6] = {hq.len, lq.len, lqn.len, main_len, un_len, unn_len};
    put("sizes", std::vector<uint8_t>(reinterpret_cast<const uint8_t*>(sizes),
                                      reinterpret_cast<const uint8_t*>(sizes) + sizeof(sizes)));
    // block statistics: reads, non-N reads, N reads, pseudogenome reads,
    // unmatched, mapped, unmapped (non-N, N), overlap passes, contested
    // suffixes, records, mismatches; overlap suffixes, and summed over the
    // passes: unlinked suffixes, suffixes probed, probes that met a prefix,
    // probes that searched a bucket, prefix comparisons; overlap links; for
    // the mapping, forward then reverse complement: reads searched, k-mer
    // probes listed, candidate windows compared; prefix rows the probes read;
    // full-match passes with both lists non-empty, and over them the summed
    // suffix and prefix list lengths
    unsigned long long mt[6] = {0, 0, 0, 0, 0, 0}, ft[3] = {0, 0, 0};
    if (mo.tally) read_small(mt, mo.tally, sizeof(mt), s);
    if (fm_tally) read_small(ft, fm_tally, sizeof(ft), s);
    const uint64_t stats[29] = {n,          m,           NN,         n_ref,         U,           n_map,
                                n_ug,       n_un,        ostats.passes, ostats.contested, n_records, n_mis,
                                ostats.suffixes, ostats.active_sum, ostats.probes, ostats.hits, ostats.searched,
                                ostats.compares, ostats.links, mt[0], mt[1], mt[2], mt[3], mt[4], mt[5],
                                ostats.rows, ft[0], ft[1], ft[2]};
    put("stats", std::vector<uint8_t>(reinterpret_cast<const uint8_t*>(stats),
                                      reinterpret_cast<const uint8_t*>(stats) + sizeof(stats)));
}

}  // namespace curc
