// a2-a5: duplicate links, k-mer index over prefix reads, error-free overlap
// linking over offsets 1..max_off-1, chain filter.
//
// Reference: compress.cu:1409-1420 (dedupe), 1427-1471 (index), 1473-1532
// (overlap passes, atomicCAS linking), 1539-1585 (filter and partition).
//
// Determinism.  The reference links with atomicCAS, so which suffix wins a
// contested prefix depends on scheduling.  Here the result is defined as the
// sequential loop over suffixes in list order, and computed in parallel
// exactly: every suffix whose equal-prefix run is claimed by it alone links
// directly (runs of different suffix strings are disjoint); suffixes that
// share a run are resolved by one thread per run, in list order.
#include "compact.cuh"
#include "stages.cuh"

namespace curc {

namespace {

__global__ void dedupe_kernel(const uint64_t* __restrict__ db, int W, const uint32_t* __restrict__ sorted, uint32_t m,
                              uint32_t* __restrict__ next, uint32_t* __restrict__ prev, uint16_t* __restrict__ offset) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i + 1 >= m) return;
    const uint32_t a = sorted[i], b = sorted[i + 1];
    const uint64_t* ra = db + uint64_t(a) * W;
    const uint64_t* rb = db + uint64_t(b) * W;
    for (int w = 0; w < W; ++w)
        if (ra[w] != rb[w]) return;
    next[a] = b;
    prev[b] = a;
    offset[a] = 0;
}

__global__ void link_flags_kernel(const uint32_t* __restrict__ sorted, uint32_t m, const uint32_t* __restrict__ next,
                                  const uint32_t* __restrict__ prev, uint8_t* __restrict__ pre_f,
                                  uint8_t* __restrict__ suf_f) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const uint32_t id = sorted[i];
    pre_f[i] = prev[id] == INVALID;
    suf_f[i] = next[id] == INVALID;
}

__global__ void prefix_hash_kernel(const uint64_t* __restrict__ db, int W, int kip, int k, uint32_t mask,
                                   uint32_t bmask, const uint32_t* __restrict__ pre, uint32_t m,
                                   uint32_t* __restrict__ keys, uint32_t* __restrict__ present) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const uint64_t hv = murmur64(word_at(db + uint64_t(pre[i]) * W, kip, k));
    keys[i] = uint32_t(hv & mask);
    const uint32_t bit = uint32_t(hv >> 32) & bmask;
    atomicOr(&present[bit >> 5], 1u << (bit & 31));
}

__global__ void gather_rows_kernel(const uint64_t* __restrict__ db, int W, const uint32_t* __restrict__ ids,
                                   uint32_t m, uint64_t* __restrict__ out) {
    const uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= uint64_t(m) * W) return;
    const uint32_t i = uint32_t(t / W), w = uint32_t(t - uint64_t(i) * W);
    out[t] = db[uint64_t(ids[i]) * W + w];
}

// keep flag of each suffix (not linked) as a 0/1 count for the scan
__global__ void keep_count_kernel(const uint8_t* __restrict__ linked, uint32_t ms, uint32_t* __restrict__ keep) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < ms) keep[j] = !linked[j];
}

// moves the kept suffixes (id, packed words, offset mask) to their
// compacted slots, preserving list order
__global__ void compact_rows_kernel(const uint32_t* __restrict__ suf, const uint64_t* __restrict__ sufw, int W,
                                    const uint32_t* __restrict__ mask, int mw, uint32_t ms, uint32_t ms2,
                                    const uint32_t* __restrict__ keep, const uint32_t* __restrict__ pos,
                                    uint32_t* __restrict__ suf2, uint64_t* __restrict__ sufw2,
                                    uint32_t* __restrict__ mask2) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= ms || !keep[j]) return;
    const uint32_t q = pos[j];
    for (int w = 0; w < W; ++w) sufw2[uint64_t(q) * W + w] = sufw[uint64_t(j) * W + w];
    for (int w = 0; w < mw; ++w) mask2[uint64_t(w) * ms2 + q] = mask[uint64_t(w) * ms + j];
    suf2[q] = suf[j];
}

__global__ void bucket_count_kernel(const uint32_t* __restrict__ keys, uint32_t m, uint32_t* __restrict__ kr) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) atomicAdd(&kr[keys[i]], 1u);
}

// bit h of bfree: bucket h still holds a prefix without a predecessor
__global__ void bucket_free_bits_kernel(const uint32_t* __restrict__ cnt, uint32_t words, uint32_t* __restrict__ bfree) {
    for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < words; w += gridDim.x * blockDim.x) {
        uint32_t v = 0;
        const uint4* c4 = reinterpret_cast<const uint4*>(cnt + uint64_t(w) * 32);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const uint4 c = c4[q];
            v |= uint32_t(c.x != 0) << (4 * q) | uint32_t(c.y != 0) << (4 * q + 1) | uint32_t(c.z != 0) << (4 * q + 2) |
                 uint32_t(c.w != 0) << (4 * q + 3);
        }
        bfree[w] = v;
    }
}

// Per prefix slot, while a pass runs: how many suffixes met the run that
// starts there, the lowest of their list indices, and the head of the list
// of their indices (one sector for the three).
struct __align__(16) RunSlot {
    uint32_t claim, lead, head, pad;
};

struct OverlapCtx {
    const uint64_t* db;
    int W, L, k, kip;
    uint32_t mask;
    const uint32_t* present;  // bitmap of prefix k-mer hashes (high 32 bits)
    uint32_t bmask;
    const uint32_t* va;  // prefix ids sorted by (bucket, read)
    const uint32_t* kr;  // bucket ranges
    uint32_t* free_cnt;  // per bucket: prefixes without a predecessor
    uint32_t* bfree;     // per bucket: free_cnt != 0 (one bit, stays in L2)
    uint32_t* next;
    uint32_t* prev;
    uint16_t* offset;
};

// First free non-self prefix of the equal run starting at lo, if equal;
// sr = the suffix read's packed words.
__device__ __forceinline__ bool link_first_free(const OverlapCtx& c, uint32_t s, const uint64_t* sr, uint32_t lo,
                                                uint32_t e, int off) {
    const int cl = c.L - off;
    for (uint32_t q = lo; q < e; ++q) {
        const uint32_t pr = c.va[q];
        if (pr == s || c.prev[pr] != INVALID) continue;
        // the probe found prefix lo equal; later entries need the comparison
        if (q == lo || cmp_span(c.db + uint64_t(pr) * c.W, 0, sr, off, cl) == 0) {
            c.prev[pr] = s;
            c.next[s] = pr;
            c.offset[s] = uint16_t(off);
            return true;
        }
        return false;
    }
    return false;
}

// A prefix of bucket h got its predecessor: the bucket's free count drops,
// and its bit clears with the last one.
__device__ __forceinline__ void take_from_bucket(const OverlapCtx& c, uint32_t h) {
    if (atomicSub(&c.free_cnt[h], 1u) == 1u) atomicAnd(&c.bfree[h >> 5], ~(1u << (h & 31)));
}

// Offsets at which a suffix can meet a prefix at all: bit off of the
// suffix's mask (word off/32 of the list's masks, stored word-major so a
// pass reads one coalesced u32 per suffix) is set when the k-mer at kmer_index_pos+off is in the
// presence bitmap of prefix k-mers.  The prefix set is fixed for the whole
// stage, so this is computed once, with the suffix's words in registers.
// Word wi of the masks (offsets 32 wi .. 32 wi + 31).  Words after the
// first are computed only when the passes reach them, for the suffixes
// still unlinked then.
__global__ void offset_mask_kernel(OverlapCtx c, const uint64_t* __restrict__ sufw, uint32_t ms, int max_off, int wi,
                                   uint32_t* __restrict__ mask) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= ms) return;
    const uint64_t* sr = sufw + uint64_t(j) * c.W;
    // 32 independent bitmap lookups in flight per thread
    uint32_t word = 0;
#pragma unroll
    for (int b = 0; b < 32; ++b) {
        const int off = wi * 32 + b;
        if (off > 0 && off < max_off) {
            const uint64_t hv = murmur64(word_at(sr, c.kip + off, c.k));
            const uint32_t bit = uint32_t(hv >> 32) & c.bmask;
            word |= ((c.present[bit >> 5] >> (bit & 31)) & 1u) << b;
        }
    }
    mask[uint64_t(wi) * ms + j] = word;
}

// The suffixes probed in a pass: not yet linked, and with a prefix k-mer
// present at this offset (mask bit).  Listing them first lets the probe and
// resolve kernels give every thread real work, instead of warps that wait on
// the few lanes whose suffix probes.
struct ProbeFilter {
    const uint8_t* linked;
    const uint32_t* mrow;  // mask word off/32 of every suffix
    uint32_t bit;
    __device__ bool operator()(uint32_t j) const { return !linked[j] && ((mrow[j] >> bit) & 1u); }
};
struct ProbeListMove {
    uint32_t* plist;
    __device__ void operator()(uint32_t j, uint32_t d) const { plist[d] = j; }
};

// Three-way compare of prefix entry `it` ([0, cl)) with the suffix's
// [off, off + cl); every comparison reads the prefix's row (counted in
// `rows`).  Prefixes of one bucket share the indexed k-mer and, for true
// overlaps, their first bases too, so a stored first word decided only a
// quarter of the comparisons and cost more than it saved.
__device__ __forceinline__ int cmp_prefix(const OverlapCtx& c, uint32_t it, const uint64_t* sr, int off, int cl,
                                          uint32_t& rows) {
    ++rows;
    return cmp_span(c.db + uint64_t(c.va[it]) * c.W, 0, sr, off, cl);
}

// compress.cu:1476-1501, the part after the hash: lower bound of
// suffix[off, L) among the prefix[0, L-off) of bucket h (whose free bit was
// set).  Returns whether an equal prefix exists; then the hit (list index,
// run start, bucket end, bucket) is set and the suffix joins the run's
// claimers.
__device__ __forceinline__ bool search_bucket(const OverlapCtx& c, const uint64_t* __restrict__ sufw, uint32_t j,
                                              uint32_t h, int off, RunSlot* __restrict__ run,
                                              uint32_t* __restrict__ gnext, uint4& hitrec, uint32_t& searched,
                                              uint32_t& compares, uint32_t& rows) {
    const int cl = c.L - off;
    const uint64_t* sr = sufw + uint64_t(j) * c.W;
    uint32_t lo = c.kr[h];
    const uint32_t e = c.kr[h + 1];
    uint32_t count = e - lo;
    ++searched;
    // lower bound; the entry it ends on (if below e) is the last one that
    // compared >= 0, so its comparison decides equality without a re-read
    int at_hi = 1;
    while (count > 0) {
        ++compares;
        const uint32_t step = count / 2, it = lo + step;
        const int r = cmp_prefix(c, it, sr, off, cl, rows);
        if (r < 0) {
            lo = it + 1;
            count -= step + 1;
        } else {
            count = step;
            at_hi = r;
        }
    }
    if (lo >= e || at_hi != 0) return false;
    // run membership: count, lowest list index, and a list of members
    atomicAdd(&run[lo].claim, 1u);
    atomicMin(&run[lo].lead, j);
    gnext[j] = atomicExch(&run[lo].head, j);
    hitrec = make_uint4(j, lo, e, h);
    return true;
}

constexpr uint32_t PROBE_THREADS = 512;

// Probes every listed suffix and lists the hits (hlist, *hcount; their
// order is immaterial to the resolution).  Two phases per block, so that
// the dependent loads of the bucket search run with full warps: every
// thread hashes one listed suffix and tests its bucket's free bit (most
// buckets have none left after the first passes), the suffixes that pass
// are queued in shared memory (one slot range per warp, from a ballot),
// and whenever a block's worth is queued, and at the end, each thread
// searches the bucket of one queued suffix.  Which thread searches which
// suffix does not change any result: a probe reads only the index and the
// free bits, which no probe of the pass writes, and the run's claim count,
// lowest member and member set do not depend on the order of the claims.
// tally[0] counts probes, tally[1] hits, tally[4] probes that searched a
// bucket, tally[5] prefix comparisons, tally[6] prefix rows read (for the
// algorithmic bytes of the pass).
__global__ void __launch_bounds__(PROBE_THREADS) probe_kernel(OverlapCtx c, const uint64_t* __restrict__ sufw,
                                                              const uint32_t* __restrict__ plist,
                                                              const uint32_t* __restrict__ pcount, int off,
                                                              RunSlot* __restrict__ run, uint32_t* __restrict__ gnext,
                                                              uint4* __restrict__ hlist, uint32_t* __restrict__ hcount,
                                                              unsigned long long* __restrict__ tally) {
    __shared__ uint4 s_hits[PROBE_THREADS];
    // queued (suffix, bucket) pairs: fewer than PROBE_THREADS are left
    // after a search round, and one round of hashing adds at most
    // PROBE_THREADS
    __shared__ uint2 s_q[2 * PROBE_THREADS];
    __shared__ uint32_t s_n, s_base, s_qn;
    uint32_t probes = 0, hits = 0, searched = 0, compares = 0, rows = 0;
    const uint32_t np = *pcount;
    const uint32_t lane = threadIdx.x & 31u;
    if (threadIdx.x == 0) s_qn = 0;
    __syncthreads();
    for (uint64_t b0 = uint64_t(blockIdx.x) * PROBE_THREADS;; b0 += uint64_t(gridDim.x) * PROBE_THREADS) {
        const bool more = b0 < np;  // the same for the whole block
        if (more) {
            const uint64_t q = b0 + threadIdx.x;
            bool keep = false;
            uint32_t j = 0, h = 0;
            if (q < np) {
                ++probes;
                j = plist[q];
                const uint64_t* sr = sufw + uint64_t(j) * c.W;
                h = uint32_t(murmur64(word_at(sr, c.kip + off, c.k)) & c.mask);
                // every prefix of the bucket has a predecessor already: no
                // link is possible for any suffix that meets it, so none
                // needs to claim it
                keep = (c.bfree[h >> 5] >> (h & 31)) & 1u;
            }
            const uint32_t bal = __ballot_sync(0xffffffffu, keep);
            uint32_t slot = 0;
            if (lane == 0 && bal) slot = atomicAdd(&s_qn, uint32_t(__popc(bal)));
            slot = __shfl_sync(0xffffffffu, slot, 0);
            if (keep) s_q[slot + uint32_t(__popc(bal & ((1u << lane) - 1u)))] = make_uint2(j, h);
            __syncthreads();
        }
        const uint32_t qn = s_qn;  // the same for the whole block (read after a barrier)
        if (qn >= PROBE_THREADS || (!more && qn > 0)) {
            // search the last `take` queued suffixes; the rest stay in place
            const uint32_t take = qn < PROBE_THREADS ? qn : PROBE_THREADS;
            bool hit = false;
            uint4 rec;
            if (threadIdx.x < take) {
                const uint2 e = s_q[qn - take + threadIdx.x];
                hit = search_bucket(c, sufw, e.x, e.y, off, run, gnext, rec, searched, compares, rows);
                hits += hit;
            }
            if (threadIdx.x == 0) s_n = 0;
            __syncthreads();
            if (threadIdx.x == 0) s_qn = qn - take;
            if (hit) s_hits[atomicAdd(&s_n, 1u)] = rec;
            __syncthreads();
            if (threadIdx.x == 0 && s_n) s_base = atomicAdd(hcount, s_n);
            __syncthreads();
            if (threadIdx.x < s_n) hlist[s_base + threadIdx.x] = s_hits[threadIdx.x];
            __syncthreads();
        }
        if (!more) break;
    }
    block_tally<unsigned long long>(probes, &tally[0]);
    block_tally<unsigned long long>(hits, &tally[1]);
    block_tally<unsigned long long>(searched, &tally[4]);
    block_tally<unsigned long long>(compares, &tally[5]);
    block_tally<unsigned long long>(rows, &tally[6]);
}

constexpr uint32_t RESOLVE_BATCH = 16;

// A suffix alone on its run links directly.  A run claimed by several
// suffixes is resolved by its lowest-index member, which visits the members
// in list order (ascending index, in sorted batches from one walk of the
// member list each) and gives each the first free non-self prefix, exactly
// the sequential loop of compress.cu:1474.  The run's bookkeeping is reset
// for the next pass by the thread that used it.  tally[2] counts links,
// tally[3] the members of contested runs.

__global__ void __launch_bounds__(512) resolve_kernel(OverlapCtx c, const uint32_t* __restrict__ suf,
                                                      const uint64_t* __restrict__ sufw,
                                                      const uint4* __restrict__ hlist,
                                                      const uint32_t* __restrict__ hcount, int off,
                                                      RunSlot* __restrict__ run, const uint32_t* __restrict__ gnext,
                                                      uint8_t* __restrict__ linked,
                                                      unsigned long long* __restrict__ tally) {
    uint32_t links = 0, contested = 0;
    const uint32_t nh = *hcount;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < nh; q += gridDim.x * blockDim.x) {
        // members of a run share its start, bucket end and bucket
        const uint4 hr = hlist[q];
        const uint32_t j = hr.x, lo = hr.y, e = hr.z, h = hr.w;
        const RunSlot rs = run[lo];
        const uint32_t n = rs.claim;
        if (n == 1) {
            if (link_first_free(c, suf[j], sufw + uint64_t(j) * c.W, lo, e, off)) {
                linked[j] = 1;
                ++links;
                take_from_bucket(c, h);
            }
        } else if (rs.lead == j) {
            // members in ascending list index: each walk of the run's member
            // list keeps the RESOLVE_BATCH smallest above the last one
            // handled, in order, so a run of n members takes
            // ceil(n / RESOLVE_BATCH) walks instead of n
            contested += n;
            uint32_t buf[RESOLVE_BATCH];
            uint32_t last = 0;
            bool first = true;
            for (;;) {
                uint32_t cnt = 0;
                for (uint32_t m = rs.head; m != INVALID; m = gnext[m]) {
                    if (!first && m <= last) continue;
                    if (cnt == RESOLVE_BATCH && m >= buf[RESOLVE_BATCH - 1]) continue;
                    uint32_t t = cnt < RESOLVE_BATCH ? cnt++ : RESOLVE_BATCH - 1;
                    while (t > 0 && buf[t - 1] > m) {
                        buf[t] = buf[t - 1];
                        --t;
                    }
                    buf[t] = m;
                }
                for (uint32_t t = 0; t < cnt; ++t) {
                    const uint32_t best = buf[t];
                    if (link_first_free(c, suf[best], sufw + uint64_t(best) * c.W, lo, e, off)) {
                        linked[best] = 1;
                        ++links;
                        take_from_bucket(c, h);
                    }
                }
                if (cnt < RESOLVE_BATCH) break;
                last = buf[RESOLVE_BATCH - 1];
                first = false;
            }
        } else {
            continue;  // the run's lowest member resolves it
        }
        run[lo] = RunSlot{0, INVALID, INVALID, 0};
    }
    block_tally<unsigned long long>(links, &tally[2]);
    block_tally<unsigned long long>(contested, &tally[3]);
}

__global__ void set_u32_kernel(uint32_t* p, uint32_t v) { *p = v; }

__global__ void run_slots_init_kernel(RunSlot* run, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) run[i] = RunSlot{0, INVALID, INVALID, 0};
}

__global__ void chain_res_kernel(uint32_t n, const uint32_t* __restrict__ next, const uint32_t* __restrict__ prev,
                                 const uint16_t* __restrict__ offset, uint8_t* __restrict__ res) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const uint32_t nx = next[r], pv = prev[r];
    uint8_t keep = 0;
    if (nx != INVALID && pv != INVALID) keep = 1;
    else if (nx != INVALID && offset[r] == 0) keep = 1;
    else if (pv != INVALID && offset[pv] == 0) keep = 1;
    res[r] = keep;
}

// A link is dropped iff one of its ends is filtered out; concurrent writers
// only ever store INVALID, so the result is schedule independent.
__global__ void chain_unlink_kernel(uint32_t n, uint32_t* next, uint32_t* prev, const uint8_t* __restrict__ res) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n || res[r]) return;
    const uint32_t nx = next[r];
    if (nx != INVALID) {
        prev[nx] = INVALID;
        next[r] = INVALID;
    }
    const uint32_t pv = prev[r];
    if (pv != INVALID) {
        next[pv] = INVALID;
        prev[r] = INVALID;
    }
}

__global__ void gather_flags_kernel(const uint32_t* __restrict__ ids, uint32_t m, const uint8_t* __restrict__ res,
                                    uint8_t* __restrict__ f, uint8_t* __restrict__ nf) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const uint8_t v = res[ids[i]];
    f[i] = v;
    nf[i] = !v;
}

inline int log2_exact(uint32_t x) {
    int b = 0;
    while ((1u << b) < x) ++b;
    return b;
}

}  // namespace

void dedupe_links(const uint64_t* db, int W, const uint32_t* sorted, uint32_t m, uint32_t* next, uint32_t* prev,
                  uint16_t* offset, cudaStream_t s) {
    if (m < 2) return;
    dedupe_kernel<<<grid_for(m, 256), 256, 0, s>>>(db, W, sorted, m, next, prev, offset);
    CURC_LAUNCH_CHECK();
}

void overlap_link(const BlockParams& p, const uint64_t* db, const uint32_t* sorted, uint32_t m, uint32_t* next,
                  uint32_t* prev, uint16_t* offset, Arena& a, cudaStream_t s, OverlapStats* st) {
    if (m == 0) return;
    auto mk = a.mark();
    uint8_t* pre_f = a.alloc<uint8_t>(m);
    uint8_t* suf_f = a.alloc<uint8_t>(m);
    link_flags_kernel<<<grid_for(m, 256), 256, 0, s>>>(sorted, m, next, prev, pre_f, suf_f);
    CURC_LAUNCH_CHECK();
    uint32_t* pre = a.alloc<uint32_t>(m);
    uint32_t* suf = a.alloc<uint32_t>(m);
    uint32_t* suf2 = a.alloc<uint32_t>(m);
    uint32_t* counts = a.alloc<uint32_t>(4);
    select_flagged(sorted, pre_f, pre, m, counts + 0, a, s);
    select_flagged(sorted, suf_f, suf, m, counts + 1, a, s);
    uint32_t hc[2];
    read_small(hc, counts, 8, s);
    const uint32_t mp = hc[0];
    uint32_t ms = hc[1];

    SubStage sp_index("overlap.index");
    // index: stable sort of prefixes by bucket (compress.cu:1440-1471)
    // The table size does not change which prefixes a suffix meets: equal
    // strings share a bucket whatever its size, and other bucket entries are
    // rejected by the comparison.  The reference sizes it to the prefix count
    // (get_hash_size); four times that keeps most probes of unlinkable
    // suffixes at one empty bucket instead of a binary search.
    const uint32_t hs = hash_size_for(uint64_t(mp) * uint64_t(p.tune.table_factor));
    // presence bitmap, 16 bits per prefix (2^20..2^32 bits): a test that stays
    // in L2 rejects most suffixes without touching the bucket table
    int bbits = 20;
    while (bbits < 32 && (1ull << bbits) < uint64_t(mp) * uint64_t(p.tune.bitmap_bits)) ++bbits;
    const uint64_t bwords = (1ull << bbits) / 32;
    uint32_t* present = a.alloc<uint32_t>(bwords);
    CURC_CHECK(cudaMemsetAsync(present, 0, bwords * 4, s));
    OverlapCtx c{db, p.W, p.L, p.k, p.kip, hs - 1, present, uint32_t((1ull << bbits) - 1), pre, nullptr, nullptr,
                 nullptr, next, prev, offset};
    uint32_t* keys = a.alloc<uint32_t>(mp ? mp : 1);
    SubStage sp_sort("overlap.index_sort");
    if (mp) {
        prefix_hash_kernel<<<grid_for(mp, 256), 256, 0, s>>>(db, p.W, p.kip, p.k, c.mask, c.bmask, pre, mp, keys,
                                                             present);
        CURC_LAUNCH_CHECK();
        radix_sort_pairs<uint32_t, uint32_t>(keys, pre, mp, 0, log2_exact(hs), a, s);
    }
    uint32_t* kr = a.alloc<uint32_t>(size_t(hs) + 2);
    CURC_CHECK(cudaMemsetAsync(kr, 0, (size_t(hs) + 2) * sizeof(uint32_t), s));
    if (mp) {
        bucket_count_kernel<<<grid_for(mp, 256), 256, 0, s>>>(keys, mp, kr);
        CURC_LAUNCH_CHECK();
    }
    uint32_t* free_cnt = a.alloc<uint32_t>(size_t(hs) + 32);
    uint32_t* bfree = a.alloc<uint32_t>(hs / 32 + 1);
    CURC_CHECK(cudaMemcpyAsync(free_cnt, kr, size_t(hs) * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
    bucket_free_bits_kernel<<<grid_for(hs / 32, 256), 256, 0, s>>>(free_cnt, hs / 32, bfree);
    CURC_LAUNCH_CHECK();
    c.free_cnt = free_cnt;
    c.bfree = bfree;
    exclusive_scan<uint32_t>(kr, kr, size_t(hs) + 2, nullptr, a, s);
    c.kr = kr;
    sp_sort.stop();

    // per prefix slot: run claim count, lowest claimer, member list head
    RunSlot* run = a.alloc<RunSlot>(mp ? mp : 1);
    run_slots_init_kernel<<<grid_for(mp ? mp : 1, 256), 256, 0, s>>>(run, mp ? mp : 1);
    CURC_LAUNCH_CHECK();
    uint32_t* gnext = a.alloc<uint32_t>(ms ? ms : 1);
    uint32_t* keepc = a.alloc<uint32_t>(ms ? ms : 1);
    uint32_t* kpos = a.alloc<uint32_t>(ms ? ms : 1);
    // suffix reads and offset masks in list order
    const int W = p.W, mw = (p.max_off + 31) / 32;
    uint64_t* sufw = a.alloc<uint64_t>(size_t(ms ? ms : 1) * W);
    uint64_t* sufw2 = a.alloc<uint64_t>(size_t(ms ? ms : 1) * W);
    uint32_t* mask = a.alloc<uint32_t>(size_t(ms ? ms : 1) * mw);
    uint32_t* mask2 = a.alloc<uint32_t>(size_t(ms ? ms : 1) * mw);
    uint8_t* linked = a.alloc<uint8_t>(ms ? ms : 1);
    CURC_CHECK(cudaMemsetAsync(linked, 0, ms ? ms : 1, s));
    SubStage sp_mask("overlap.index_mask");
    if (ms) {
        gather_rows_kernel<<<grid_for(uint64_t(ms) * W, 256), 256, 0, s>>>(db, W, suf, ms, sufw);
        CURC_LAUNCH_CHECK();
        if (mp) {
            offset_mask_kernel<<<grid_for(ms, 256), 256, 0, s>>>(c, sufw, ms, p.max_off, 0, mask);
            CURC_LAUNCH_CHECK();
        }
    }
    sp_mask.stop();
    // probes, probes that met a prefix, links, contested members
    unsigned long long* tally = a.alloc<unsigned long long>(7);
    CURC_CHECK(cudaMemsetAsync(tally, 0, 56, s));
    sp_index.stop();

    // List of size ms, of which `active` are unlinked; compacted once half
    // of it has linked.  Passes are queued without a host round trip; the
    // host reads the link count every few passes to compact or stop.
    uint32_t* plist = a.alloc<uint32_t>(ms ? ms : 1);
    uint4* hlist = a.alloc<uint4>(ms ? ms : 1);
    uint32_t* hcount = a.alloc<uint32_t>(p.max_off + 1);  // one per pass
    CURC_CHECK(cudaMemsetAsync(hcount, 0, size_t(p.max_off + 1) * 4, s));
    uint32_t* dcount = a.alloc<uint32_t>(2);  // [0] list size, [1] listed probes
    set_u32_kernel<<<1, 1, 0, s>>>(dcount, ms);
    CURC_LAUNCH_CHECK();
    Compactor cp(ms, a, s);
    const int gp = resident_grid(probe_kernel, PROBE_THREADS, ms ? ms : 1);
    const int gr = resident_grid(resolve_kernel, 512, ms ? ms : 1);
    const int CHECK_EVERY = p.tune.check_every;
    uint32_t passes = 0, active = ms;
    uint64_t links_seen = 0, active_sum = 0;
    const uint32_t ms0 = ms;
    int words = 1;  // mask words computed so far
    auto compact = [&] {
        SubStage sp_comp("overlap.compact");
        const int g = grid_for(ms, 256);
        keep_count_kernel<<<g, 256, 0, s>>>(linked, ms, keepc);
        CURC_LAUNCH_CHECK();
        exclusive_scan<uint32_t>(keepc, kpos, ms, nullptr, a, s);
        compact_rows_kernel<<<g, 256, 0, s>>>(suf, sufw, W, mask, words, ms, active, keepc, kpos, suf2, sufw2, mask2);
        CURC_LAUNCH_CHECK();
        std::swap(suf, suf2);
        std::swap(sufw, sufw2);
        std::swap(mask, mask2);
        ms = active;
        CURC_CHECK(cudaMemsetAsync(linked, 0, ms ? ms : 1, s));
        set_u32_kernel<<<1, 1, 0, s>>>(dcount, ms);
        CURC_LAUNCH_CHECK();
    };
    for (int off = 1; off < p.max_off && active > 0 && mp > 0; ++off) {
        if ((off >> 5) >= words) {  // next mask word, for the unlinked suffixes only
            const uint64_t links = read_scalar(tally + 2, s);
            active -= uint32_t(links - links_seen);
            links_seen = links;
            if (active < ms) compact();
            if (ms) {
                SubStage sp_mw("overlap.index_mask");
                offset_mask_kernel<<<grid_for(ms, 256), 256, 0, s>>>(c, sufw, ms, p.max_off, words, mask);
                CURC_LAUNCH_CHECK();
            }
            ++words;
            if (active == 0) break;
        }
        ++passes;
        active_sum += active;  // as of the last check
        SubStage sp_probe("overlap.probe_resolve");
        SubStage sp_filter("overlap.filter");
        cp.run(dcount, ms, dcount + 1,
               ProbeFilter{linked, mask + uint64_t(off >> 5) * ms, uint32_t(off & 31)}, ProbeListMove{plist});
        sp_filter.stop();
        SubStage sp_pk("overlap.probe");
        probe_kernel<<<gp, PROBE_THREADS, 0, s>>>(c, sufw, plist, dcount + 1, off, run, gnext,
                                        hlist, hcount + off, tally);
        CURC_LAUNCH_CHECK();
        sp_pk.stop();
        SubStage sp_rk("overlap.resolve");
        resolve_kernel<<<gr, 512, 0, s>>>(c, suf, sufw, hlist, hcount + off, off, run,
                                          gnext, linked, tally);
        CURC_LAUNCH_CHECK();
        sp_rk.stop();
        sp_probe.stop();
        if (off % CHECK_EVERY != 0 && off + 1 < p.max_off) continue;
        const uint64_t links = read_scalar(tally + 2, s);
        active -= uint32_t(links - links_seen);
        links_seen = links;
        if (active * 2 < ms) compact();
    }
    cp.check();
    if (st) {
        unsigned long long t[7];
        read_small(t, tally, 56, s);
        st->passes = passes;
        st->links = uint32_t(t[2]);
        st->contested = uint32_t(t[3]);
        st->suffixes = ms0;
        st->active_sum = active_sum;
        st->probes = t[0];
        st->hits = t[1];
        st->searched = t[4];
        st->compares = t[5];
        st->rows = t[6];
    }
    a.release(mk);
}

void chain_filter(uint32_t n, const uint32_t* sorted, uint32_t m, uint32_t* next, uint32_t* prev,
                  const uint16_t* offset, uint32_t* ref_ids, uint32_t* unmatch_ids, uint32_t* counts, Arena& a,
                  cudaStream_t s) {
    // compress.cu:1539-1572
    auto mk = a.mark();
    uint8_t* res = a.alloc<uint8_t>(n ? n : 1);
    if (n) {
        chain_res_kernel<<<grid_for(n, 256), 256, 0, s>>>(n, next, prev, offset, res);
        CURC_LAUNCH_CHECK();
        chain_unlink_kernel<<<grid_for(n, 256), 256, 0, s>>>(n, next, prev, res);
        CURC_LAUNCH_CHECK();
    }
    uint8_t* f = a.alloc<uint8_t>(m ? m : 1);
    uint8_t* nf = a.alloc<uint8_t>(m ? m : 1);
    if (m) {
        gather_flags_kernel<<<grid_for(m, 256), 256, 0, s>>>(sorted, m, res, f, nf);
        CURC_LAUNCH_CHECK();
    }
    select_flagged(sorted, f, ref_ids, m, counts + 0, a, s);
    select_flagged(sorted, nf, unmatch_ids, m, counts + 1, a, s);
    a.release(mk);
}

}  // namespace curc
