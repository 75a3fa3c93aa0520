// Stage entry points of the device pipeline (host-callable, stream-ordered).
// Every array argument is a device pointer unless stated otherwise.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "common.cuh"
#include "primitives.cuh"

namespace curc {

std::string& ctxless_error();

// Launch and table choices that change no result (the autotuner's knobs):
// the overlap index's bucket table size as a multiple of the prefix count
// (the reference's get_hash_size is factor 1; equal strings share a bucket
// whatever the size), bits of the prefix presence bitmap per prefix, how
// many overlap passes run between host reads of the link count, and the
// threads per block of the mapping kernel (one warp per read).
struct Tuning {
    int table_factor = 4, bitmap_bits = 16, check_every = 8, map_threads = 128;
    int fm_loop = 1;  // full-match pass loop: 0 a launch per kernel, 1 one graph, 2 one persistent kernel
};

// Autotuner cache key of a block: read length and read count rounded down
// to a power of two.
struct TuneKey {
    int L, log2n;
    bool operator<(const TuneKey& o) const { return L != o.L ? L < o.L : log2n < o.log2n; }
};
inline TuneKey tune_key(int L, uint64_t n) {
    int b = 0;
    while (b < 63 && (uint64_t(1) << (b + 1)) <= n) ++b;
    return TuneKey{L, b};
}

struct BlockParams {
    int L = 0, W = 0, max_off = 0, k = 0, kip = 0, max_mm = 0;
    bool preserve_order = false, paired_end = false;
    Tuning tune;
    static BlockParams derive(int L, bool po, bool pe) {  // preprocess.cpp:295-313
        BlockParams p;
        p.L = L;
        p.W = (L + 31) / 32;
        p.max_off = L * 65 / 100;
        p.k = L < 89 ? 36 * L / 100 : 32;
        p.kip = L - p.k - p.max_off;
        p.max_mm = L / 5;
        p.preserve_order = po;
        p.paired_end = pe;
        return p;
    }
    static constexpr int bucket_limit = 12, k1 = 28, ref_step = 5, read_step = 2, target_mm = 1;
};

// AlignmentRecord (compress.cu:68-77) as laid out on the device.
struct DevRecord {
    uint32_t read_id;
    uint8_t is_n, strand;
    uint16_t pad;
    uint64_t pos;
};
static_assert(sizeof(DevRecord) == 16, "record layout");

// ---- a1 (pack.cu)
void pack_reads(const uint8_t* seq, uint64_t n, int L, uint64_t* packed, uint8_t* has_n, uint32_t* err,
                cudaStream_t s);
void split_n_reads(const uint8_t* has_n, uint64_t n, uint32_t* reads_id, uint32_t* n_reads_id, uint32_t* counts,
                   Arena& a, cudaStream_t s);
void gather_ascii_rows(const uint8_t* seq, const uint32_t* ids, uint32_t m, int L, uint8_t* out, cudaStream_t s);

// ---- a2..a5 (overlap.cu)
void dedupe_links(const uint64_t* db, int W, const uint32_t* sorted, uint32_t m, uint32_t* next, uint32_t* prev,
                  uint16_t* offset, cudaStream_t s);
struct OverlapStats {
    uint32_t passes = 0, links = 0, contested = 0, suffixes = 0;
    uint64_t active_sum = 0, probes = 0, hits = 0, searched = 0, compares = 0, rows = 0;  // summed over passes
};
void overlap_link(const BlockParams& p, const uint64_t* db, const uint32_t* sorted, uint32_t m, uint32_t* next,
                  uint32_t* prev, uint16_t* offset, Arena& a, cudaStream_t s, OverlapStats* st = nullptr);
// res flags + unlink; writes ref ids and unmatched ids (sorted order) and
// their counts to counts[0], counts[1].
void chain_filter(uint32_t n, const uint32_t* sorted, uint32_t m, uint32_t* next, uint32_t* prev,
                  const uint16_t* offset, uint32_t* ref_ids, uint32_t* unmatch_ids, uint32_t* counts, Arena& a,
                  cudaStream_t s);

// ---- a6/a7 (fullmatch.cu)
// Packed reads: prefix/suffix lists are consumed (scratch).  tally (device,
// 3 counters, optional): passes with both lists non-empty, and their summed
// suffix and prefix list lengths.
void full_match_packed(const BlockParams& p, const uint64_t* db, uint32_t* pre, uint32_t* suf, uint32_t cnt,
                       uint32_t* next, uint32_t* prev, uint16_t* offset, Arena& a, cudaStream_t s,
                       unsigned long long* tally = nullptr);
// ASCII reads (N reads): sorts `ids` (count m) by content, links exact
// duplicates, then runs the suffix-prefix merge.  next/prev/offset have
// n_total entries and are initialised here.
void full_match_ascii(const BlockParams& p, const uint8_t* reads, uint32_t* ids, uint32_t m, uint32_t n_total,
                      uint32_t* next, uint32_t* prev, uint16_t* offset, Arena& a, cudaStream_t s);
void sort_ids_by_ascii(const uint8_t* reads, int L, uint32_t* ids, uint32_t m, Arena& a, cudaStream_t s);

// ---- a8 (assembly.cu)
struct Assembled {
    DevRecord* records = nullptr;   // one per member read, chain order
    uint32_t n_records = 0;
    uint8_t* seq = nullptr;         // ASCII pseudogenome
    uint64_t len = 0;
    uint64_t* packed = nullptr;     // 2-bit copy + one zero pad word
};
// Reads are packed (db, W) when ascii == nullptr, else ASCII rows of length L.
void assemble(const uint64_t* db, const uint8_t* ascii, int L, int W, const uint32_t* ids, uint32_t m,
              uint32_t n_total, const uint32_t* next, const uint32_t* prev, const uint16_t* offset, bool is_n,
              Assembled& out, Arena& a, cudaStream_t s);
void pack_ascii_ref(const uint8_t* seq, uint64_t len, uint64_t* packed, cudaStream_t s);

// ---- a9 (mapper.cu)
struct MapOut {
    uint8_t* mm = nullptr;       // per read (U then N)
    uint8_t* strand = nullptr;
    uint64_t* pos = nullptr;
    // optional counters, forward then reverse complement: reads searched,
    // k-mer probes listed, candidate windows compared
    unsigned long long* tally = nullptr;
};
void map_reads(const BlockParams& p, const uint64_t* ref, uint64_t ref_len, const uint64_t* udb, uint32_t U,
               const uint8_t* ndb, uint32_t NN, MapOut& out, Arena& a, cudaStream_t s);

void gather_packed_rows(const uint64_t* db, int W, const uint32_t* ids, uint32_t m, uint64_t* out, cudaStream_t s);

}  // namespace curc
