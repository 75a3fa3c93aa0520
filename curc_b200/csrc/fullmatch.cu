// a6/a7: exact suffix-prefix merge of chain ends over every offset.
//
// Reference: full_match_gpu compress.cu:1003-1174 (packed reads) and
// full_match_cpu compress.cu:1176-1347 (ASCII N reads, alphabet ACGNT).
//
// Per offset the reference (1) re-sorts the suffix list by read[off, L) with
// a split on base off-1 and stable merges, (2) buckets both lists by a
// 10-base (3-symbol for ASCII) prefix with 4^10 binary searches, and (3)
// runs one sequential two-pointer merge per bucket.  Inside a bucket the
// merge pairs, in order, the suffixes and prefixes of each run of equal
// strings (with a rotation when a read meets itself), so here the work is
// organised per run of equal suffix strings instead: no fixed 4^10 cost,
// and one thread per run executes the reference's merge steps for that run.
//
// (1) is done as a tree of parallel stable pairwise merges of the
// per-symbol runs (merge path).
#include "compact.cuh"
#include "stages.cuh"

namespace curc {

namespace {

struct PackedAcc {
    const uint64_t* db;
    int W, L;
    static constexpr int ALPHA = 4;
    __device__ __forceinline__ int cmp(uint32_t a, int aoff, uint32_t b, int boff, int len) const {
        return cmp_span(db + uint64_t(a) * W, aoff, db + uint64_t(b) * W, boff, len);
    }
    __device__ __forceinline__ int sym(uint32_t a, int pos) const { return code_at(db + uint64_t(a) * W, pos); }
    // key: the first KS symbols of read a from pos, left-aligned, zero padded
    static constexpr int KS = 32, SB = 2;
    __device__ __forceinline__ uint64_t key(uint32_t a, int pos) const {
        const int nb = L - pos < KS ? L - pos : KS;
        return word_at(db + uint64_t(a) * W, uint32_t(pos), nb) << (64 - SB * nb);
    }
};

struct AsciiAcc {
    const uint8_t* r;
    int W, L;  // W unused
    static constexpr int ALPHA = 5;
    __device__ __forceinline__ int cmp(uint32_t a, int aoff, uint32_t b, int boff, int len) const {
        const uint8_t* x = r + uint64_t(a) * L + aoff;
        const uint8_t* y = r + uint64_t(b) * L + boff;
        for (int i = 0; i < len; ++i)
            if (x[i] != y[i]) return x[i] < y[i] ? -1 : 1;
        return 0;
    }
    // partition symbols of compress.cu:1238-1249: A, C, G, N, everything else
    __device__ __forceinline__ int sym(uint32_t a, int pos) const {
        switch (r[uint64_t(a) * L + pos]) {
            case 'A': return 0;
            case 'C': return 1;
            case 'G': return 2;
            case 'N': return 3;
            default: return 4;
        }
    }
    static constexpr int KS = 8, SB = 8;
    __device__ __forceinline__ uint64_t key(uint32_t a, int pos) const {
        const uint8_t* x = r + uint64_t(a) * L;
        uint64_t v = 0;
        for (int b = 0; b < KS; ++b) v = (v << 8) | (pos + b < L ? x[pos + b] : 0);
        return v;
    }
};

// Comparison of read a from aoff with read b from boff over len symbols,
// given their keys at those offsets (the key comparison decides unless the
// first KS symbols are equal and more follow).
template <class Acc>
__device__ __forceinline__ int cmp_keyed(const Acc& acc, uint64_t ka, uint32_t a, int aoff, uint64_t kb, uint32_t b,
                                         int boff, int len) {
    if (len < Acc::KS) {
        const uint64_t mask = ~0ull << (64 - Acc::SB * len);
        ka &= mask;
        kb &= mask;
    }
    if (ka != kb) return ka < kb ? -1 : 1;
    if (len <= Acc::KS) return 0;
    return acc.cmp(a, aoff + Acc::KS, b, boff + Acc::KS, len - Acc::KS);
}

// The pass's offset: a kernel argument when the host queues the passes,
// read from device memory when the passes replay from a graph.
struct FmOff {
    int v;
    const int* p;
    __device__ __forceinline__ int get() const { return p ? *p : v; }
};

// Keys of the list entries [t0, m) step ts at offset off.  With sym_count
// (2-bit reads only), also how many entries have each base at off-1: the
// list is sorted by read[off-1, L), so these counts give the base runs'
// bounds.  Each thread counts in four 16-bit fields (a resident grid leaves
// it far fewer than 65536 entries), then one atomic per block and base
// (every thread of the block calls this).
template <class Acc>
__device__ __forceinline__ void list_keys_range(const Acc& acc, const uint32_t* __restrict__ ids, uint32_t m, int off,
                                                uint64_t* __restrict__ key, uint32_t* __restrict__ sym_count,
                                                uint32_t t0, uint32_t ts) {
    uint64_t c = 0;
    for (uint32_t i = t0; i < m; i += ts) {
        const uint32_t id = ids[i];
        key[i] = acc.key(id, off);
        if constexpr (Acc::ALPHA == 4)
            if (sym_count) c += 1ull << (16 * acc.sym(id, off - 1));
    }
    if constexpr (Acc::ALPHA == 4)
        if (sym_count)
            for (int b = 0; b < 4; ++b) block_tally<uint32_t>(uint32_t(c >> (16 * b)) & 0xFFFFu, sym_count + b);
}

// With tally: one thread adds the pass to the counters (passes with both
// lists non-empty, their suffix and prefix entries; mp_dev is the prefix
// list's length).
template <class Acc>
__global__ void list_keys_kernel(Acc acc, const uint32_t* __restrict__ ids, const uint32_t* __restrict__ m_dev,
                                 FmOff fo, uint64_t* __restrict__ key, uint32_t* __restrict__ sym_count,
                                 const uint32_t* __restrict__ mp_dev, unsigned long long* __restrict__ tally) {
    const uint32_t m = *m_dev;
    const int off = fo.get();
    if (tally && blockIdx.x == 0 && threadIdx.x == 0) {
        const uint32_t mp = *mp_dev;
        if (m && mp) {
            tally[0] += 1;
            tally[1] += m;
            tally[2] += mp;
        }
    }
    list_keys_range(acc, ids, m, off, key, sym_count, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

// bounds[c] = first index whose symbol at off-1 is >= c (the list is
// sorted by read[off-1, L), so symbols are nondecreasing).  One block
// narrows all boundaries at once, 64 threads each: every round samples 64
// evenly spaced positions of the boundary's interval, so a few rounds of
// independent loads replace a chain of ~log2(m) dependent ones.
// (One block of at least 256 threads; every thread calls it.)
template <class Acc>
__device__ __forceinline__ void run_bounds_block(const Acc& acc, const uint32_t* __restrict__ suf, uint32_t m, int off,
                                                 uint32_t* __restrict__ bounds) {
    constexpr int NB = Acc::ALPHA - 1;  // boundaries to find: symbols 1 .. ALPHA-1 (at most 4)
    constexpr uint32_t S = 64;          // samples per boundary and round
    __shared__ uint32_t lo_s[4], hi_s[4];
    __shared__ uint8_t sym_s[4][S];
    const int b = int(threadIdx.x / S);
    const uint32_t t = threadIdx.x % S;
    // invariant for boundary b: indices < lo have symbol < b+1, indices >= hi
    // have symbol >= b+1
    if (threadIdx.x < 4) {
        lo_s[threadIdx.x] = 0;
        hi_s[threadIdx.x] = m;
    }
    __syncthreads();
    for (;;) {
        bool open = false;
#pragma unroll
        for (int q = 0; q < NB; ++q) open |= lo_s[q] < hi_s[q];
        if (!open) break;
        const uint32_t lo = b < NB ? lo_s[b] : 0, hi = b < NB ? hi_s[b] : 0;
        const uint32_t span = hi - lo, k = span < S ? span : S;
        if (b < NB && t < k) sym_s[b][t] = uint8_t(acc.sym(suf[lo + uint32_t((uint64_t(span) * t) / k)], off - 1));
        __syncthreads();
        if (b < NB && t == 0 && lo < hi) {
            uint32_t f = 0;  // first sample with symbol >= b+1
            while (f < k && sym_s[b][f] < uint32_t(b + 1)) ++f;
            const uint32_t pf = f < k ? lo + uint32_t((uint64_t(span) * f) / k) : hi;
            const uint32_t pp = f > 0 ? lo + uint32_t((uint64_t(span) * (f - 1)) / k) + 1 : lo;
            lo_s[b] = k == span ? pf : pp;  // all positions sampled: exact
            hi_s[b] = pf;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        bounds[0] = 0;
        bounds[Acc::ALPHA] = m;
    }
    if (threadIdx.x < NB) bounds[threadIdx.x + 1] = lo_s[threadIdx.x];
}

template <class Acc>
__global__ void __launch_bounds__(256) run_bounds_kernel(Acc acc, const uint32_t* __restrict__ suf,
                                                         const uint32_t* __restrict__ m_dev, FmOff fo,
                                                         uint32_t* __restrict__ bounds) {
    run_bounds_block(acc, suf, *m_dev, fo.get(), bounds);
}

// Stable merge of the symbol runs by read[off, L), as a tree of pairwise
// merges of adjacent runs (level l merges groups of 2^l runs; ties go to the
// lower run, as in the reference's stable merges), each
// output element placed by merge path: a thread takes MP_ITEMS consecutive
// outputs, finds by bisection how many of them precede in each of the two
// inputs, and then merges sequentially.  About log2(n) / MP_ITEMS + 1
// comparisons per output and level, instead of a binary search per run.
// The entries' keys at off travel with them, so a comparison reads the
// reads themselves only when the first key symbols are equal.
constexpr int MP_ITEMS = 8;

// Outputs [t0, m) step ts (in units of MP_ITEMS).
template <class Acc>
__device__ __forceinline__ void merge_level_range(const Acc& acc, int off, const uint32_t* __restrict__ in,
                                                  const uint64_t* __restrict__ ink, uint32_t* __restrict__ out,
                                                  uint64_t* __restrict__ outk, const uint32_t* __restrict__ bounds,
                                                  bool counts, uint32_t m, int width, uint64_t t0, uint64_t ts) {
    uint32_t bd[Acc::ALPHA + 1];
    if (counts) {
        bd[0] = 0;
#pragma unroll
        for (int c = 0; c < Acc::ALPHA - 1; ++c) bd[c + 1] = bd[c] + bounds[c];
        bd[Acc::ALPHA] = m;
    } else {
#pragma unroll
        for (int c = 0; c <= Acc::ALPHA; ++c) bd[c] = bounds[c];
    }
    const int len = acc.L - off;
    auto run_at = [&](int r) { return bd[r < Acc::ALPHA ? r : Acc::ALPHA]; };
    // entry x against entry y (positions in the input)
    auto cmp_at = [&](uint32_t x, uint32_t y) {
        return cmp_keyed(acc, ink[x], in[x], off, ink[y], in[y], off, len);
    };
    const uint64_t stride = ts * MP_ITEMS;
    for (uint64_t d0 = t0 * MP_ITEMS; d0 < m; d0 += stride) {
        const uint32_t dend = uint32_t(min(uint64_t(m), d0 + MP_ITEMS));
        uint32_t d = uint32_t(d0);
        int k = 0;
        while (d < dend) {
            // the pair of run groups that holds output d
            uint32_t a0 = run_at(2 * k * width), a1 = run_at((2 * k + 1) * width), a2 = run_at((2 * k + 2) * width);
            while (d >= a2) {
                ++k;
                a0 = run_at(2 * k * width);
                a1 = run_at((2 * k + 1) * width);
                a2 = run_at((2 * k + 2) * width);
            }
            const uint32_t na = a1 - a0, nb = a2 - a1, dd = d - a0;
            uint32_t lo = dd > nb ? dd - nb : 0, hi = dd < na ? dd : na;
            while (lo < hi) {
                const uint32_t mid = (lo + hi) / 2;
                if (cmp_at(a0 + mid, a1 + dd - mid - 1) <= 0)
                    lo = mid + 1;
                else
                    hi = mid;
            }
            uint32_t i = lo, j = dd - lo;
            const uint32_t stop = dend < a2 ? dend : a2;
            for (; d < stop; ++d) {
                const bool take_a = j >= nb || (i < na && cmp_at(a0 + i, a1 + j) <= 0);
                const uint32_t x = take_a ? a0 + i++ : a1 + j++;
                out[d] = in[x];
                outk[d] = ink[x];
            }
        }
    }
}

// bounds: the run bounds (ALPHA + 1 entries), or with `counts` the number of
// entries per symbol, from which the bounds are summed.
template <class Acc>
__global__ void merge_level_kernel(Acc acc, FmOff fo, const uint32_t* __restrict__ in, const uint64_t* __restrict__ ink,
                                   uint32_t* __restrict__ out, uint64_t* __restrict__ outk,
                                   const uint32_t* __restrict__ bounds, bool counts, const uint32_t* __restrict__ m_dev,
                                   int width) {
    merge_level_range(acc, fo.get(), in, ink, out, outk, bounds, counts, *m_dev, width,
                      uint64_t(blockIdx.x) * blockDim.x + threadIdx.x, uint64_t(gridDim.x) * blockDim.x);
}

// One thread per run of equal suffix strings: the reference's bucket merge
// restricted to that run (compress.cu:1089-1160 / 1297-1336).  Prefix keys
// (at offset 0) and suffix keys (at off) decide most comparisons.
template <class Acc>
__device__ __forceinline__ void group_one(const Acc& acc, uint32_t* pre, uint64_t* pk, uint32_t mp,
                                          const uint32_t* __restrict__ suf, const uint64_t* __restrict__ sk,
                                          uint32_t ms, int off, uint32_t j, uint32_t* next, uint32_t* prev,
                                          uint16_t* offset) {
    const int len = acc.L - off;
    const uint32_t s0 = suf[j];
    const uint64_t k0 = sk[j];
    if (j > 0 && cmp_keyed(acc, sk[j - 1], suf[j - 1], off, k0, s0, off, len) == 0) return;
    // prefixes P with P[0, len) == s0[off, L)
    auto pcmp = [&](uint32_t i) { return cmp_keyed(acc, pk[i], pre[i], 0, k0, s0, off, len); };
    uint32_t lo = 0, count = mp;
    while (count > 0) {
        uint32_t step = count / 2, it = lo + step;
        if (pcmp(it) < 0) {
            lo = it + 1;
            count -= step + 1;
        } else {
            count = step;
        }
    }
    uint32_t hi = lo;
    while (hi < mp && pcmp(hi) == 0) ++hi;
    if (hi == lo) return;
    uint32_t se = j + 1;
    while (se < ms && cmp_keyed(acc, sk[se], suf[se], off, k0, s0, off, len) == 0) ++se;
    uint32_t pi = lo, si = j;
    while (pi < hi && si < se) {
        uint32_t P = pre[pi];
        const uint32_t S = suf[si];
        if (P == S) {
            const uint32_t cur = pi;
            bool found = false;
            while (pi + 1 < hi) {
                ++pi;
                if (pre[pi] != S) {
                    found = true;
                    break;
                }
            }
            if (!found) {
                pi = cur;
                ++si;
                continue;
            }
            // rotate P to the front of [cur, pi], keys alongside
            P = pre[pi];
            const uint64_t K = pk[pi];
            while (pi > cur) {
                pre[pi] = pre[pi - 1];
                pk[pi] = pk[pi - 1];
                --pi;
            }
            pre[pi] = P;
            pk[pi] = K;
        }
        next[S] = P;
        prev[P] = S;
        offset[S] = uint16_t(off);
        ++pi;
        ++si;
    }
}

template <class Acc>
__global__ void merge_groups_kernel(Acc acc, uint32_t* pre, uint64_t* pk, const uint32_t* __restrict__ mp_dev,
                                    const uint32_t* __restrict__ suf, const uint64_t* __restrict__ sk,
                                    const uint32_t* __restrict__ ms_dev, FmOff fo, uint32_t* next, uint32_t* prev,
                                    uint16_t* offset) {
    const uint32_t mp = *mp_dev, ms = *ms_dev;
    if (mp == 0) return;
    const int off = fo.get();
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < ms; j += gridDim.x * blockDim.x)
        group_one(acc, pre, pk, mp, suf, sk, ms, off, j, next, prev, offset);
}

// ---------------------------------------------------------------- persistent form
//
// One cooperative launch runs every pass: the phases of a pass (keys and
// run bounds, the merge levels, the pairing, a two-phase compaction of both
// lists) are separated by grid-wide barriers instead of kernel boundaries,
// and the lists' lengths are read from device memory at the top of each
// pass, so neither launches nor host reads separate the passes.  Every block
// is resident (cooperative launch), which the barriers need.  The results
// are those of the launch-per-kernel form: the same device functions do the
// work, and the compaction keeps both lists in order (chunks in block order,
// entries in index order inside a chunk).
constexpr int FM_THREADS = 256;
constexpr uint32_t FM_BARRIER_LIMIT = 1u << 22;  // ~0.3 s of 64 ns sleeps; a barrier takes microseconds

// Grid-wide barrier with a bounded wait (cooperative launch: every block
// resident).  word[0] counts arrivals, word[1] is the generation, word[2]
// the error flag.  Block writes before the barrier are visible to every
// block after it (block barrier, then a device-scope fence by the arriving
// thread, and one after the wait).  Returns false once any block's wait
// has run out: the caller leaves the loop, so no block waits for ever.
__device__ __forceinline__ bool fm_grid_barrier(uint32_t* word, uint32_t nblocks) {
    __shared__ uint32_t s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile uint32_t* gen = word + 1;
        volatile uint32_t* err = word + 2;
        const uint32_t g = *gen;
        __threadfence();
        bool ok = *err == 0;
        if (ok) {
            if (atomicAdd(word, 1u) == nblocks - 1) {
                word[0] = 0;
                __threadfence();
                atomicAdd(word + 1, 1u);
            } else {
                uint32_t spins = 0;
                while (*gen == g) {
                    if (*err != 0 || ++spins > FM_BARRIER_LIMIT) {
                        atomicExch(word + 2, 1u);
                        ok = false;
                        break;
                    }
                    __nanosleep(64);
                }
            }
        }
        __threadfence();
        s_ok = ok ? 1u : 0u;
    }
    __syncthreads();
    return s_ok != 0;
}

struct FmPersist {
    uint32_t *pre, *tmp, *suf, *suf2, *mtmp;
    uint64_t *pk, *tk, *sk, *sk2, *mk2;
    uint32_t* bounds;             // run bounds, or base counts (2-bit reads; zero at launch)
    uint32_t* len;                // [0] prefixes, [1] suffixes in the lists
    uint32_t* bcnt;               // per block: kept prefixes, then kept suffixes (2 x gridDim)
    uint32_t *next, *prev;
    uint16_t* offset;
    unsigned long long* tally;    // optional: passes, suffix and prefix entries
    uint32_t* passes;             // passes run
    uint32_t* barrier;            // fm_grid_barrier words (3; zero at launch)
};

// Block-wide exclusive scan of one value per thread (FM_THREADS threads);
// returns the thread's exclusive prefix, *total the block's sum.
__device__ __forceinline__ uint32_t fm_block_scan(uint32_t v, uint32_t* s_warp, uint32_t* total) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t incl = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t u = __shfl_up_sync(0xFFFFFFFFu, incl, d);
        if (lane >= uint32_t(d)) incl += u;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    uint32_t before = 0, all = 0;
#pragma unroll
    for (int w = 0; w < FM_THREADS / 32; ++w) {
        const uint32_t c = s_warp[w];
        before += w < int(warp) ? c : 0;
        all += c;
    }
    __syncthreads();  // s_warp is reused by the next call
    *total = all;
    return before + incl - v;
}

// Block-wide sum (FM_THREADS threads).
__device__ __forceinline__ uint32_t fm_block_sum(uint32_t v, uint32_t* s_warp) {
    uint32_t t;
    fm_block_scan(v, s_warp, &t);
    return t;
}

template <class Acc>
__global__ void __launch_bounds__(FM_THREADS) fm_persistent_kernel(Acc acc, FmPersist st) {
    __shared__ uint32_t s_warp[FM_THREADS / 32];
    auto sync = [&] { return fm_grid_barrier(st.barrier, gridDim.x); };
    constexpr bool by_count = Acc::ALPHA == 4;
    int levels = 0;
    while ((1 << levels) < Acc::ALPHA) ++levels;
    const uint32_t G = gridDim.x;
    const uint64_t gt = uint64_t(blockIdx.x) * FM_THREADS + threadIdx.x, gs = uint64_t(G) * FM_THREADS;
    uint32_t* pre = st.pre;
    uint32_t* tmp = st.tmp;
    uint64_t* pk = st.pk;
    uint64_t* tk = st.tk;
    uint32_t passes = 0;
    for (int off = 1; off < acc.L; ++off) {
        // the lengths were written before the last barrier; read past L1 so
        // that every block sees the same values and takes the same barriers
        const uint32_t mp = *reinterpret_cast<volatile const uint32_t*>(st.len);
        const uint32_t ms = *reinterpret_cast<volatile const uint32_t*>(st.len + 1);
        if (mp == 0 || ms == 0) break;
        ++passes;
        if (gt == 0 && st.tally) {
            st.tally[0] += 1;
            st.tally[1] += ms;
            st.tally[2] += mp;
        }
        // keys of the suffixes at off (and, 2-bit reads, their base counts at off-1)
        list_keys_range(acc, st.suf, ms, off, st.sk, by_count ? st.bounds : nullptr, uint32_t(gt), uint32_t(gs));
        if (!by_count && blockIdx.x == 0) run_bounds_block(acc, st.suf, ms, off, st.bounds);
        if (!sync()) break;
        // merge levels: the last one writes suf2/sk2
        bool alive = true;
        {
            const uint32_t* src = st.suf;
            const uint64_t* srck = st.sk;
            for (int l = 0; l < levels && alive; ++l) {
                const bool last = l + 1 == levels;
                uint32_t* dst = last ? st.suf2 : (l % 2 == 0 ? st.mtmp : st.suf);
                uint64_t* dstk = last ? st.sk2 : (l % 2 == 0 ? st.mk2 : st.sk);
                merge_level_range(acc, off, src, srck, dst, dstk, st.bounds, by_count, ms, 1 << l, gt, gs);
                alive = sync();
                src = dst;
                srck = dstk;
            }
        }
        if (!alive) break;
        // pairing, one thread per run of equal suffix strings
        for (uint64_t j = gt; j < ms; j += gs)
            group_one(acc, pre, pk, mp, st.suf2, st.sk2, ms, off, uint32_t(j), st.next, st.prev, st.offset);
        if (by_count && gt < 4) st.bounds[gt] = 0;  // counts of the next pass (the merges are done)
        if (!sync()) break;
        // compaction, phase 1: kept entries of this block's chunk of each list
        const uint32_t cp = (mp + G - 1) / G, cs = (ms + G - 1) / G;
        const uint32_t p0 = min(mp, blockIdx.x * cp), p1 = min(mp, p0 + cp);
        const uint32_t s0 = min(ms, blockIdx.x * cs), s1 = min(ms, s0 + cs);
        {
            uint32_t kp = 0, ks = 0;
            for (uint32_t i = p0 + threadIdx.x; i < p1; i += FM_THREADS) kp += st.prev[pre[i]] == INVALID;
            for (uint32_t i = s0 + threadIdx.x; i < s1; i += FM_THREADS) ks += st.next[st.suf2[i]] == INVALID;
            kp = fm_block_sum(kp, s_warp);
            ks = fm_block_sum(ks, s_warp);
            if (threadIdx.x == 0) {
                st.bcnt[blockIdx.x] = kp;
                st.bcnt[G + blockIdx.x] = ks;
            }
        }
        if (!sync()) break;
        // phase 2: this chunk's place from the chunks before it, then the
        // kept entries in order
        {
            uint32_t bp = 0, bs = 0, tp = 0, ts = 0;
            const volatile uint32_t* bc = st.bcnt;  // other blocks' counts, from L2
            for (uint32_t b = threadIdx.x; b < G; b += FM_THREADS) {
                const uint32_t a = bc[b], c = bc[G + b];
                tp += a;
                ts += c;
                if (b < blockIdx.x) {
                    bp += a;
                    bs += c;
                }
            }
            bp = fm_block_sum(bp, s_warp);
            bs = fm_block_sum(bs, s_warp);
            tp = fm_block_sum(tp, s_warp);
            ts = fm_block_sum(ts, s_warp);
            for (uint32_t i0 = p0; i0 < p1; i0 += FM_THREADS) {
                const uint32_t i = i0 + threadIdx.x;
                const bool keep = i < p1 && st.prev[pre[i]] == INVALID;
                uint32_t tile;
                const uint32_t r = fm_block_scan(keep ? 1u : 0u, s_warp, &tile);
                if (keep) {
                    tmp[bp + r] = pre[i];
                    tk[bp + r] = pk[i];
                }
                bp += tile;
            }
            for (uint32_t i0 = s0; i0 < s1; i0 += FM_THREADS) {
                const uint32_t i = i0 + threadIdx.x;
                const bool keep = i < s1 && st.next[st.suf2[i]] == INVALID;
                uint32_t tile;
                const uint32_t r = fm_block_scan(keep ? 1u : 0u, s_warp, &tile);
                if (keep) st.suf[bs + r] = st.suf2[i];
                bs += tile;
            }
            if (gt == 0) {
                st.len[0] = tp;
                st.len[1] = ts;
            }
        }
        uint32_t* t32 = pre;
        pre = tmp;
        tmp = t32;
        uint64_t* t64 = pk;
        pk = tk;
        tk = t64;
        if (!sync()) break;
    }
    if (gt == 0) *st.passes = passes;
}

// Compaction functors: keep the list entries whose link is still free.
struct FreeLink {
    const uint32_t* ids;
    const uint32_t* link;
    __device__ bool operator()(uint32_t i) const { return link[ids[i]] == INVALID; }
};
struct MoveId {
    const uint32_t* in;
    uint32_t* out;
    __device__ void operator()(uint32_t i, uint32_t d) const { out[d] = in[i]; }
};
struct MoveIdKey {
    const uint32_t* in;
    const uint64_t* ink;
    uint32_t* out;
    uint64_t* outk;
    __device__ void operator()(uint32_t i, uint32_t d) const {
        out[d] = in[i];
        outk[d] = ink[i];
    }
};

__global__ void fm_zero4_kernel(uint32_t* p) { p[threadIdx.x] = 0; }

// Graph form of the pass loop.  After the first pass of a replayed pair the
// offset advances; past the last offset the second pass's list lengths are
// zeroed, so its launches find no work.
__global__ void fm_step_kernel(int* offp, uint32_t* next_len, int L) {
    const int o = ++*offp;
    if (o >= L) {
        next_len[0] = 0;
        next_len[1] = 0;
    }
}

// After the second pass: the device loop goes on while offsets remain and
// both lists hold entries.  The offset grows by two per iteration, so the
// loop ends after at most L / 2 iterations whatever the lists hold; the
// iteration count is capped at L as well, independently of the offset.
__global__ void fm_cond_kernel(cudaGraphConditionalHandle h, int* offp, const uint32_t* len, int L,
                               uint32_t* iters) {
    const int o = ++*offp;
    const uint32_t it = ++*iters;
    cudaGraphSetConditional(h, (o < L && it < uint32_t(L) && len[0] != 0 && len[1] != 0) ? 1u : 0u);
}

// The passes run without a host round trip: list lengths stay on the
// device (two slots per list, read by one pass and written by its
// compaction) and kernels walk them with resident grids.  Three forms, with
// the same results (tune.fm_loop): 0, one launch per kernel from the host,
// which looks at the lengths every few passes to stop early (and times the
// sub-stages); 1, a graph whose conditional `while` node replays a pair of
// passes, the offset and the stop test on the device, so one graph launch
// runs the whole loop; 2, one persistent cooperative kernel whose phases
// are separated by grid-wide barriers (fm_persistent_kernel).
template <class Acc>
void full_match_loop(const Acc& acc, uint32_t* pre, uint32_t* suf, uint32_t cnt, uint32_t* next, uint32_t* prev,
                     uint16_t* offset, int mode, unsigned long long* tally, Arena& a, cudaStream_t s) {
    // nothing to link without ends; a single prefix and a single suffix can
    // still link when they are different reads (the head and the tail of one
    // chain, which then closes into a cycle, as the reference's merge does)
    if (cnt == 0 || acc.L < 2) return;
    if (cnt == 1) {  // one end of each kind: nothing links when both are the same read
        uint32_t ends[2];
        read_small(ends, pre, 4, s);
        read_small(ends + 1, suf, 4, s);
        if (ends[0] == ends[1]) return;
    }
    auto mk = a.mark();
    uint32_t* suf2 = a.alloc<uint32_t>(cnt);
    uint32_t* tmp = a.alloc<uint32_t>(cnt);
    uint32_t* mtmp = a.alloc<uint32_t>(cnt);
    // keys: prefixes at offset 0 (kept with the prefix list), suffixes at
    // the pass's offset (taken at the start of each pass)
    uint64_t* pk = a.alloc<uint64_t>(cnt);
    uint64_t* tk = a.alloc<uint64_t>(cnt);
    uint64_t* sk = a.alloc<uint64_t>(cnt);
    uint64_t* sk2 = a.alloc<uint64_t>(cnt);
    uint64_t* mk2 = a.alloc<uint64_t>(cnt);
    uint32_t* bounds = a.alloc<uint32_t>(8);
    uint32_t* len = a.alloc<uint32_t>(4);  // mp, ms for even passes, then for odd passes
    int* offp = a.alloc<int>(2);           // graph form: [0] the pass's offset, [1] iterations
    const uint32_t init[4] = {cnt, cnt, 0, 0};
    CURC_CHECK(cudaMemcpyAsync(len, init, sizeof(init), cudaMemcpyHostToDevice, s));
    Compactor cp(cnt, a, s);
    const int gk = resident_grid(list_keys_kernel<Acc>, 256, cnt);
    const int gm = resident_grid(merge_level_kernel<Acc>, 256, div_up(cnt, MP_ITEMS));
    const int gg = resident_grid(merge_groups_kernel<Acc>, 128, cnt);
    list_keys_kernel<Acc><<<gk, 256, 0, s>>>(acc, pre, len, FmOff{0, nullptr}, pk, nullptr, nullptr, nullptr);
    CURC_LAUNCH_CHECK();
    // 2-bit reads: the base runs' bounds come from counts taken with the keys
    constexpr bool by_count = Acc::ALPHA == 4;

    // One pass over the lists in slots `par`, at offset fo.
    auto pass = [&](FmOff fo, int par, bool graph) {
        uint32_t* mp_in = len + 2 * par;
        uint32_t* ms_in = mp_in + 1;
        uint32_t* mp_out = len + 2 * (par ^ 1);
        uint32_t* ms_out = mp_out + 1;
        SubStage sp_merge("full_match.resort", !graph);
        if (by_count) {
            if (graph) {  // a kernel node rather than a memset node in the loop body
                fm_zero4_kernel<<<1, 4, 0, s>>>(bounds);
                CURC_LAUNCH_CHECK();
            } else {
                CURC_CHECK(cudaMemsetAsync(bounds, 0, 4 * sizeof(uint32_t), s));
            }
        } else {
            run_bounds_kernel<Acc><<<1, 256, 0, s>>>(acc, suf, ms_in, fo, bounds);
            CURC_LAUNCH_CHECK();
        }
        list_keys_kernel<Acc><<<gk, 256, 0, s>>>(acc, suf, ms_in, fo, sk, by_count ? bounds : nullptr, mp_in,
                                                  tally);
        CURC_LAUNCH_CHECK();
        {
            // levels: runs merged in pairs, then pairs of pairs, ...; the last
            // level writes suf2/sk2 (suf/sk are free after the first level)
            int levels = 0;
            while ((1 << levels) < Acc::ALPHA) ++levels;
            const uint32_t* src = suf;
            const uint64_t* srck = sk;
            for (int l = 0; l < levels; ++l) {
                const bool last = l + 1 == levels;
                uint32_t* dst = last ? suf2 : (l % 2 == 0 ? mtmp : suf);
                uint64_t* dstk = last ? sk2 : (l % 2 == 0 ? mk2 : sk);
                merge_level_kernel<Acc><<<gm, 256, 0, s>>>(acc, fo, src, srck, dst, dstk, bounds, by_count, ms_in,
                                                            1 << l);
                CURC_LAUNCH_CHECK();
                src = dst;
                srck = dstk;
            }
        }
        sp_merge.stop();
        SubStage sp_groups("full_match.groups", !graph);
        merge_groups_kernel<Acc><<<gg, 128, 0, s>>>(acc, pre, pk, mp_in, suf2, sk2, ms_in, fo, next, prev, offset);
        CURC_LAUNCH_CHECK();
        sp_groups.stop();
        SubStage sp_comp("full_match.compact", !graph);
        if (graph) {
            cp.run_replayable(mp_in, cnt, mp_out, FreeLink{pre, prev}, MoveIdKey{pre, pk, tmp, tk});
            cp.run_replayable(ms_in, cnt, ms_out, FreeLink{suf2, next}, MoveId{suf2, suf});
        } else {
            cp.run(mp_in, cnt, mp_out, FreeLink{pre, prev}, MoveIdKey{pre, pk, tmp, tk});
            cp.run(ms_in, cnt, ms_out, FreeLink{suf2, next}, MoveId{suf2, suf});
        }
        std::swap(pre, tmp);
        std::swap(pk, tk);
        sp_comp.stop();
    };

    if (mode == 2) {
        SubStage sp_loop("full_match.persistent");
        int dev = 0, sms = 0, per_sm = 0;
        CURC_CHECK(cudaGetDevice(&dev));
        CURC_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        CURC_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fm_persistent_kernel<Acc>, FM_THREADS, 0));
        if (per_sm < 1) throw std::runtime_error("full match: the persistent kernel does not fit on an SM");
        const int grid = sms * per_sm;  // every block resident: the barriers need it
        uint32_t* bcnt = a.alloc<uint32_t>(2 * size_t(grid));
        uint32_t* barrier = a.alloc<uint32_t>(4);
        CURC_CHECK(cudaMemsetAsync(bounds, 0, 8 * sizeof(uint32_t), s));
        CURC_CHECK(cudaMemsetAsync(barrier, 0, 4 * sizeof(uint32_t), s));
        FmPersist fp{pre,  tmp,  suf,  suf2,   mtmp,  pk,    tk,                                  sk,
                     sk2,  mk2,  bounds, len,  bcnt,  next,  prev,                                offset,
                     tally, reinterpret_cast<uint32_t*>(offp), barrier};
        Acc acc_arg = acc;
        void* args[] = {&acc_arg, &fp};
        CURC_CHECK(cudaLaunchCooperativeKernel(reinterpret_cast<void*>(fm_persistent_kernel<Acc>), grid, FM_THREADS,
                                               args, 0, s));
        CURC_LAUNCH_CHECK();
        sp_loop.stop();
        uint32_t err = 0;
        read_small(&err, barrier + 2, 4, s);
        if (err) throw std::runtime_error("full match: a grid barrier wait of the persistent kernel ran out");
    } else if (mode == 0) {
        constexpr int CHECK_EVERY = 8;
        int par = 0;
        for (int off = 1; off < acc.L; ++off, par ^= 1) {
            pass(FmOff{off, nullptr}, par, false);
            if (off % CHECK_EVERY == 0) {
                uint32_t h[2];
                read_small(h, len + 2 * (par ^ 1), 8, s);
                if (h[0] == 0 || h[1] == 0) break;
            }
        }
        cp.check();
    } else {
        SubStage sp_loop("full_match.graph");
        const int init_off[2] = {1, 0};
        CURC_CHECK(cudaMemcpyAsync(offp, init_off, sizeof(init_off), cudaMemcpyHostToDevice, s));
        cudaGraph_t g = nullptr, body = nullptr;
        cudaGraphExec_t ge = nullptr;
        uint64_t body_launches = 0;
        try {
            CURC_CHECK(cudaGraphCreate(&g, 0));
            cudaGraphConditionalHandle h;
            CURC_CHECK(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
            cudaGraphNodeParams np = {};
            np.type = cudaGraphNodeTypeConditional;
            np.conditional.handle = h;
            np.conditional.type = cudaGraphCondTypeWhile;
            np.conditional.size = 1;
            cudaGraphNode_t node;
            CURC_CHECK(cudaGraphAddNode(&node, g, nullptr, 0, &np));
            body = np.conditional.phGraph_out[0];
            CURC_CHECK(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
            try {
                pass(FmOff{0, offp}, 0, true);
                fm_step_kernel<<<1, 1, 0, s>>>(offp, len + 2, acc.L);
                CURC_LAUNCH_CHECK();
                pass(FmOff{0, offp}, 1, true);
                fm_cond_kernel<<<1, 1, 0, s>>>(h, offp, len, acc.L, reinterpret_cast<uint32_t*>(offp + 1));
                CURC_LAUNCH_CHECK();
            } catch (...) {
                cudaGraph_t dummy = nullptr;
                cudaStreamEndCapture(s, &dummy);
                if (dummy && dummy != body) cudaGraphDestroy(dummy);
                throw;
            }
            CURC_CHECK(cudaStreamEndCapture(s, &body));
            size_t nodes = 0;  // every node of the body is a kernel
            CURC_CHECK(cudaGraphGetNodes(body, nullptr, &nodes));
            body_launches = nodes;
            CURC_CHECK(cudaGraphInstantiate(&ge, g, 0));
            CURC_CHECK(cudaGraphLaunch(ge, s));
        } catch (...) {
            if (ge) cudaGraphExecDestroy(ge);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        sp_loop.stop();
        cp.check();  // synchronises: the graph has run
        uint32_t iters = 0;
        read_small(&iters, offp + 1, 4, s);
        CURC_CHECK(cudaGraphExecDestroy(ge));
        CURC_CHECK(cudaGraphDestroy(g));
        // the captured launches were counted once; the device replayed them
        if (iters > 1) count_launches(body_launches * (iters - 1));
    }
    a.release(mk);
}

__global__ void ascii_chunk_kernel(const uint8_t* __restrict__ r, int L, const uint32_t* __restrict__ ids, uint32_t m,
                                   int chunk, uint64_t* __restrict__ key) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const uint8_t* p = r + uint64_t(ids[i]) * L + chunk * 8;
    uint64_t v = 0;
    for (int b = 0; b < 8; ++b) v = (v << 8) | (chunk * 8 + b < L ? p[b] : 0);
    key[i] = v;
}

__global__ void ascii_dedupe_kernel(const uint8_t* __restrict__ r, int L, const uint32_t* __restrict__ ids, uint32_t m,
                                    uint32_t* next, uint32_t* prev, uint16_t* offset) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i + 1 >= m) return;
    const uint32_t a = ids[i], b = ids[i + 1];
    const uint8_t* x = r + uint64_t(a) * L;
    const uint8_t* y = r + uint64_t(b) * L;
    for (int t = 0; t < L; ++t)
        if (x[t] != y[t]) return;
    prev[b] = a;
    next[a] = b;
    offset[a] = 0;
}

__global__ void ends_flags_kernel(const uint32_t* __restrict__ ids, uint32_t m, const uint32_t* __restrict__ next,
                                  const uint32_t* __restrict__ prev, uint8_t* __restrict__ pf, uint8_t* __restrict__ sf) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    pf[i] = prev[ids[i]] == INVALID;
    sf[i] = next[ids[i]] == INVALID;
}

}  // namespace

void full_match_packed(const BlockParams& p, const uint64_t* db, uint32_t* pre, uint32_t* suf, uint32_t cnt,
                       uint32_t* next, uint32_t* prev, uint16_t* offset, Arena& a, cudaStream_t s,
                       unsigned long long* tally) {
    full_match_loop(PackedAcc{db, p.W, p.L}, pre, suf, cnt, next, prev, offset, p.tune.fm_loop, tally, a, s);
}

void sort_ids_by_ascii(const uint8_t* reads, int L, uint32_t* ids, uint32_t m, Arena& a, cudaStream_t s) {
    // stable lexicographic (memcmp) order: LSD over 8-byte big-endian chunks
    if (m <= 1) return;
    auto mk = a.mark();
    uint64_t* key = a.alloc<uint64_t>(m);
    const int chunks = (L + 7) / 8;
    for (int c = chunks - 1; c >= 0; --c) {
        ascii_chunk_kernel<<<grid_for(m, 256), 256, 0, s>>>(reads, L, ids, m, c, key);
        CURC_LAUNCH_CHECK();
        const int lo = (c == chunks - 1) ? 8 * (8 * chunks - L) : 0;
        radix_sort_pairs<uint64_t, uint32_t>(key, ids, m, lo, 64, a, s);
    }
    a.release(mk);
}

void full_match_ascii(const BlockParams& p, const uint8_t* reads, uint32_t* ids, uint32_t m, uint32_t n_total,
                      uint32_t* next, uint32_t* prev, uint16_t* offset, Arena& a, cudaStream_t s) {
    // compress.cu:1179-1210: sort, duplicate links, prefix/suffix lists
    fill<uint32_t>(next, INVALID, n_total, s);
    fill<uint32_t>(prev, INVALID, n_total, s);
    fill<uint16_t>(offset, INVALOFF, n_total, s);
    if (m == 0) return;
    sort_ids_by_ascii(reads, p.L, ids, m, a, s);
    if (m > 1) {
        ascii_dedupe_kernel<<<grid_for(m, 256), 256, 0, s>>>(reads, p.L, ids, m, next, prev, offset);
        CURC_LAUNCH_CHECK();
    }
    auto mk = a.mark();
    uint8_t* pf = a.alloc<uint8_t>(m);
    uint8_t* sf = a.alloc<uint8_t>(m);
    ends_flags_kernel<<<grid_for(m, 256), 256, 0, s>>>(ids, m, next, prev, pf, sf);
    CURC_LAUNCH_CHECK();
    uint32_t* pre = a.alloc<uint32_t>(m);
    uint32_t* suf = a.alloc<uint32_t>(m);
    uint32_t* counts = a.alloc<uint32_t>(2);
    select_flagged(ids, pf, pre, m, counts + 0, a, s);
    select_flagged(ids, sf, suf, m, counts + 1, a, s);
    const uint32_t cnt = read_scalar(counts + 0, s);
    full_match_loop(AsciiAcc{reads, 0, p.L}, pre, suf, cnt, next, prev, offset, p.tune.fm_loop, nullptr, a, s);
    a.release(mk);
}

}  // namespace curc
