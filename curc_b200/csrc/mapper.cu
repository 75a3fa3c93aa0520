// a9: map leftover reads onto the pseudogenome.
//
// Reference: ReadMapper compress.cu:268-595 with util.cuh:233-270.
// A sampled index of 28-mers every 5 positions (forward, then reverse
// complemented for the second strand), buckets capped at 12 entries; each
// read probes its 28-mers at every 2nd offset and keeps the first candidate
// that strictly improves its mismatch count, stopping at <= 1 mismatch.
//
// Canonical index.  The reference fills buckets with non-atomic uint8
// counters; here a bucket holds the first 12 sampled positions in ascending
// order, stored in descending slots (the sequential outcome of
// compress.cu:368-406).  It is built with a stable radix sort of (hash,
// sample) pairs: each sample finds its rank in its bucket by looking back at
// most 12 places, so no per-bucket atomics are needed.
#include "stages.cuh"

namespace curc {

namespace {

__global__ void sample_hash_kernel(const uint64_t* __restrict__ ref, uint64_t start, uint64_t count, int k, int step,
                                   bool rc, uint32_t mask, uint32_t* __restrict__ hv, uint32_t* __restrict__ idx) {
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += uint64_t(gridDim.x) * blockDim.x) {
        uint64_t km = word_unaligned(ref, start + i * step, k);
        if (rc) km = revcomp_kmer(km, k);
        hv[i] = uint32_t(murmur64(km) & mask);
        idx[i] = uint32_t(i);
    }
}

__global__ void bucket_caps_kernel(const uint32_t* __restrict__ hv, uint64_t count, uint32_t* __restrict__ cnt) {
    for (uint64_t j = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < count; j += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t h = hv[j];
        if (j > 0 && hv[j - 1] == h) continue;
        uint32_t c = 1;
        while (c < BlockParams::bucket_limit && j + c < count && hv[j + c] == h) ++c;
        cnt[h] = c;
    }
}

__global__ void bucket_fill_kernel(const uint32_t* __restrict__ hv, const uint32_t* __restrict__ idx, uint64_t count,
                                   const uint32_t* __restrict__ kr, uint32_t* __restrict__ pos) {
    for (uint64_t j = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < count; j += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t h = hv[j];
        uint32_t rank = 0;
        while (rank < BlockParams::bucket_limit && rank < j && hv[j - 1 - rank] == h) ++rank;
        const uint32_t b = kr[h], c = kr[h + 1] - b;
        if (rank < c) pos[b + c - 1 - rank] = idx[j];
    }
}

struct MapIndex {
    uint32_t mask;
    const uint32_t* kr;
    const uint32_t* pos;
    uint64_t start;
};

// Chunk q (bases 32q .. 32q + nb - 1) of the read as compared with the
// pseudogenome: the read's own word, or for the reverse-complement strand
// the reverse complement of the matching bases from the read's end.
template <bool RC>
__device__ __forceinline__ uint64_t read_chunk(const uint64_t* __restrict__ rd, int L, int q) {
    const int i = 32 * q, nb = L - i < 32 ? L - i : 32;
    return RC ? revcomp_kmer(word_at(rd, L - i - nb, nb), nb) : word_at(rd, i, nb);
}

// util.cuh:233-270: 32-base chunks, early exit once the bound is reached.
// rw: the read's chunks (read_chunk), computed once per read.
__device__ __forceinline__ int packed_mismatches(const uint64_t* __restrict__ ref, uint64_t mp,
                                                 const uint64_t* rw, int L, int bound) {
    int c = 0;
    for (int i = 0, q = 0; i < L && c < bound; i += 32, ++q) {
        const int nb = L - i < 32 ? L - i : 32;
        c += base_mismatches(word_unaligned(ref, mp + i, nb), rw[q]);
    }
    return c;
}

template <bool RC>
__device__ __forceinline__ int ascii_mismatches(const uint64_t* __restrict__ ref, uint64_t mp,
                                                const uint8_t* __restrict__ nd, int L, int bound) {
    int c = 0;
    for (int o = 0; o < L; ++o) {
        const char rb = "ACGT"[code_at(ref, mp + o)];
        const char qb = RC ? comp_char(char(nd[L - 1 - o])) : char(nd[o]);
        if (rb != qb && ++c >= bound) break;
    }
    return c;
}

// One warp per read.  The reference's loop visits the candidates of the
// read's probes in order (probe offset, then bucket slot), takes each that
// strictly improves the mismatch count, and stops at the first count
// <= target.  So its result is the first candidate with count <= target,
// or else the first candidate with the smallest count (when that improves
// on the read's count so far).  The warp lists the candidates of 32 probes
// at a time, evaluates them 32 at a time in that order, and stops after the
// chunk in which a count <= target appears.  A candidate's count is exact
// below the smallest count met so far (the bound of the early exit, as in
// the reference's loop; the same in every lane, and above target while the
// loop runs), which is all the comparison needs: a candidate matters only
// if it reaches target or strictly improves on that count.
// One read per warp; returns (in every lane) the probes listed and the
// candidates compared for the algorithmic-byte counters.
template <bool RC>
__device__ __forceinline__ void map_read(const MapIndex& ix, const uint64_t* __restrict__ ref, uint64_t ref_len,
                                         const uint64_t* __restrict__ udb, uint32_t U,
                                         const uint8_t* __restrict__ ndb, int L, int W, int k, int step,
                                         uint8_t* __restrict__ mm, uint8_t* __restrict__ strand,
                                         uint64_t* __restrict__ pos, uint32_t i, uint32_t lane, uint32_t& listed,
                                         uint32_t& compared, uint64_t* rw) {
    const int init = mm[i];
    if (init <= BlockParams::target_mm) return;
    const bool isn = i >= U;
    const uint64_t* rd = isn ? nullptr : udb + uint64_t(i) * W;
    const uint8_t* nd = isn ? ndb + uint64_t(i - U) * L : nullptr;
    // the read's comparison words, once for all its candidates
    if (!isn && int(lane) < W) rw[lane] = read_chunk<RC>(rd, L, int(lane));
    __syncwarp();
    const int probes = (L - k) / BlockParams::read_step + 1;
    int best = init;  // smallest count met so far (the same in every lane)
    uint64_t best_pos = 0;
    bool done = false;
    for (int p0 = 0; p0 < probes && !done; p0 += 32) {
        // this lane's probe: bucket range of its k-mer
        const int pj = p0 + int(lane);
        const int j = pj * BlockParams::read_step;
        uint32_t b = 0, cnt = 0;
        if (pj < probes) {
            uint64_t key;
            if (!isn) {
                key = word_at(rd, j, k);
            } else {
                key = 0;
                for (int t = 0; t < k; ++t) key = (key << 2) | uint64_t(ascii_code(nd[j + t]));
            }
            const uint32_t h = uint32_t(murmur64(key) & ix.mask);
            b = ix.kr[h];
            const uint32_t e = ix.kr[h + 1];
            cnt = min(e - b, uint32_t(BlockParams::bucket_limit));
        }
        // inclusive scan of the candidate counts over the lanes
        uint32_t incl = cnt;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, d);
            if (lane >= uint32_t(d)) incl += v;
        }
        const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
        listed += uint32_t(min(32, probes - p0));
        for (uint32_t cs = 0; cs < total; cs += 32) {
            compared += min(32u, total - cs);
            const uint32_t ci = cs + lane;
            int c = 0x7FFF;
            uint64_t mp = 0;
            // owner lane: the first lane whose inclusive count exceeds ci
            uint32_t owner = 0;
#pragma unroll
            for (int d = 16; d > 0; d >>= 1) {
                const uint32_t v = __shfl_sync(0xFFFFFFFFu, incl, owner + d - 1);
                if (v <= ci) owner += d;
            }
            const uint32_t ob = __shfl_sync(0xFFFFFFFFu, b, owner);
            const uint32_t oex = __shfl_sync(0xFFFFFFFFu, incl - cnt, owner);
            if (ci < total) {
                const int oj = (p0 + int(owner)) * BlockParams::read_step;
                const uint32_t q = ob + (ci - oex);
                const uint64_t refpos = ix.start + uint64_t(ix.pos[q]) * step;
                const uint64_t shift = RC ? uint64_t(L - k - oj) : uint64_t(oj);
                if (refpos >= shift && refpos - shift + L <= ref_len) {
                    mp = refpos - shift;
                    // the window of the best count so far (met again through
                    // another probe) has that count, which neither reaches
                    // target nor improves: not compared again
                    if (!(best < init && mp == best_pos))
                        c = isn ? ascii_mismatches<RC>(ref, mp, nd, L, best) : packed_mismatches(ref, mp, rw, L, best);
                }
            }
            // the loop stops at the first count <= target
            const uint32_t stop = __ballot_sync(0xFFFFFFFFu, c <= BlockParams::target_mm);
            if (stop) {
                const int first = __ffs(stop) - 1;
                best = __shfl_sync(0xFFFFFFFFu, c, first);
                best_pos = __shfl_sync(0xFFFFFFFFu, mp, first);
                done = true;
                break;
            }
            // otherwise the earliest candidate of the chunk with the smallest
            // count, kept only if it strictly improves
            int cmin = c;
#pragma unroll
            for (int d = 16; d > 0; d >>= 1) cmin = min(cmin, __shfl_xor_sync(0xFFFFFFFFu, cmin, d));
            const int first = __ffs(__ballot_sync(0xFFFFFFFFu, c == cmin)) - 1;
            const uint64_t fpos = __shfl_sync(0xFFFFFFFFu, mp, first);
            if (cmin < best) {
                best = cmin;
                best_pos = fpos;
            }
        }
    }
    if (lane == 0 && best < init) {
        mm[i] = uint8_t(best);
        strand[i] = RC ? 1 : 0;
        pos[i] = best_pos;
    }
}

template <bool RC>
__global__ void __launch_bounds__(256) map_kernel(MapIndex ix, const uint64_t* __restrict__ ref, uint64_t ref_len,
                                                  const uint64_t* __restrict__ udb, uint32_t U,
                                                  const uint8_t* __restrict__ ndb, uint32_t NN, int L, int W, int k,
                                                  int step, uint8_t* __restrict__ mm, uint8_t* __restrict__ strand,
                                                  uint64_t* __restrict__ pos, unsigned long long* __restrict__ tally) {
    __shared__ uint64_t s_rw[256 / 32][16];  // per warp: the read's comparison words
    const uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t listed = 0, compared = 0;
    const bool searched = i < U + NN && mm[i] > BlockParams::target_mm;
    if (i < U + NN)  // whole warp
        map_read<RC>(ix, ref, ref_len, udb, U, ndb, L, W, k, step, mm, strand, pos, i, lane, listed, compared,
                     s_rw[threadIdx.x >> 5]);
    if (tally) {  // lane 0 carries its warp's counts
        block_tally<unsigned long long>(lane == 0 && searched ? 1u : 0u, &tally[0]);
        block_tally<unsigned long long>(lane == 0 ? listed : 0u, &tally[1]);
        block_tally<unsigned long long>(lane == 0 ? compared : 0u, &tally[2]);
    }
}

inline int log2_exact(uint32_t x) {
    int b = 0;
    while ((1u << b) < x) ++b;
    return b;
}

}  // namespace

void map_reads(const BlockParams& p, const uint64_t* ref, uint64_t ref_len, const uint64_t* udb, uint32_t U,
               const uint8_t* ndb, uint32_t NN, MapOut& out, Arena& a, cudaStream_t s) {
    const uint32_t total = U + NN;
    fill<uint8_t>(out.mm, uint8_t(p.max_mm + 1), total, s);
    fill<uint8_t>(out.strand, 0, total, s);
    fill<uint64_t>(out.pos, 0, total, s);
    const int k = BlockParams::k1, step = BlockParams::ref_step;
    if (total == 0 || ref_len < uint64_t(k)) return;
    const uint64_t index_count = (ref_len - k + 1 + step - 1) / step;
    struct Part { uint64_t start, count; };
    Part parts[2];
    int np = 1;
    if (index_count > (1ull << 30)) {  // compress.cu:342-353
        const uint64_t h = index_count / 2;
        parts[0] = {0, h};
        parts[1] = {h * step, index_count - h};
        np = 2;
    } else {
        parts[0] = {0, index_count};
    }
    for (int rc = 0; rc < 2; ++rc) {
        for (int q = 0; q < np; ++q) {
            auto mk = a.mark();
            SubStage sp_index(rc ? "mapping.index_rc" : "mapping.index_fwd");
            const uint64_t count = parts[q].count;
            const uint32_t hs = hash_size_for(count);
            uint32_t* hv = a.alloc<uint32_t>(count);
            uint32_t* idx = a.alloc<uint32_t>(count);
            sample_hash_kernel<<<grid_for(count, 256, 4), 256, 0, s>>>(ref, parts[q].start, count, k, step, rc != 0,
                                                                       hs - 1, hv, idx);
            CURC_LAUNCH_CHECK();
            radix_sort_pairs<uint32_t, uint32_t>(hv, idx, count, 0, log2_exact(hs), a, s);
            uint32_t* kr = a.alloc<uint32_t>(size_t(hs) + 2);
            CURC_CHECK(cudaMemsetAsync(kr, 0, (size_t(hs) + 2) * 4, s));
            bucket_caps_kernel<<<grid_for(count, 256, 4), 256, 0, s>>>(hv, count, kr);
            CURC_LAUNCH_CHECK();
            exclusive_scan<uint32_t>(kr, kr, size_t(hs) + 2, nullptr, a, s);
            uint32_t* pos = a.alloc<uint32_t>(std::min<uint64_t>(count, uint64_t(hs) * 12) + 2);
            bucket_fill_kernel<<<grid_for(count, 256, 4), 256, 0, s>>>(hv, idx, count, kr, pos);
            CURC_LAUNCH_CHECK();
            sp_index.stop();
            SubStage sp_map(rc ? "mapping.map_rc" : "mapping.map_fwd");
            MapIndex ix{hs - 1, kr, pos, parts[q].start};
            const int mt = p.tune.map_threads;
            const int g = grid_for(uint64_t(total) * 32, mt);
            unsigned long long* t = out.tally ? out.tally + 3 * rc : nullptr;
            if (rc)
                map_kernel<true><<<g, mt, 0, s>>>(ix, ref, ref_len, udb, U, ndb, NN, p.L, p.W, k, step, out.mm,
                                                  out.strand, out.pos, t);
            else
                map_kernel<false><<<g, mt, 0, s>>>(ix, ref, ref_len, udb, U, ndb, NN, p.L, p.W, k, step, out.mm,
                                                   out.strand, out.pos, t);
            CURC_LAUNCH_CHECK();
            a.release(mk);
        }
    }
}

}  // namespace curc
