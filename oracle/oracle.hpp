// CPU oracle for the CURC pseudogenome path -- TEST INFRASTRUCTURE ONLY.
//
// A sequential restatement of CURC's block compressor (src/compress.cu and
// src/util.cuh of the reference) used as the checker for the CUDA path.  Only
// tests, the smoke check and bench.py's CPU-baseline leg may call it.
//
// Canonical semantics.  Where the reference runs data-parallel code whose
// result depends on thread scheduling (atomicCAS overlap linking,
// non-atomic uint8 bucket counters), this oracle runs the same loop body
// sequentially in index order; sorts are stable with ties in input order.
// That is "each Thrust for_each executed in index order".
#pragma once
#include <cstdint>
#include <cstddef>
#include <string>
#include <vector>

namespace oracle {

constexpr uint32_t INVALID = 0xFFFFFFFFu;   // constant.hpp:48
constexpr uint16_t INVALOFF = 0xFFFFu;      // constant.hpp:49

// Derived block parameters (preprocess.cpp:295-313, Param.hpp:72-73).
struct Params {
    int read_len = 0;           // L
    int unit = 0;               // W = ceil(L/32) packed u64 words per read
    int max_off = 0;            // L*65/100
    int kmer_size = 0;          // 32, or 36*L/100 when L < 89
    int kmer_index_pos = 0;     // L - k - max_off
    int max_mismatch = 0;       // L/5
    bool preserve_order = false;
    bool paired_end = false;
    int flzma2_level = 10;
    int flzma2_threads = 16;
    static constexpr int bucket_limit = 12, k1 = 28, ref_step = 5, read_step = 2, target_mm = 1;
    static Params derive(int L, bool po, bool pe);
};

struct Record {                 // AlignmentRecord, compress.cu:68-77
    uint32_t read_id;
    uint8_t is_n;
    uint8_t strand;
    uint64_t pos;
};

// ---- bit helpers (util.cuh:82-281) ----
uint64_t murmur64(uint64_t x);
uint32_t hash_size_for(size_t items);
uint64_t word_at(const uint64_t* read, uint64_t off, int nbases);          // extract_word
uint64_t word_unaligned(const uint64_t* bits, uint64_t off, int nbases);   // extract_word_unaligned
char base_at(const uint64_t* bits, uint64_t off);                          // extract_base
uint64_t revcomp_kmer(uint64_t kmer, int k);                               // get_reverse_kmer
char comp_base(char b);                                                    // reverse_dna_base
uint64_t kmer_from_ascii(const char* s, int k);                            // get_kmer_integer

// ---- stages ----
// a1: 2-bit pack (compress.cu:2159-2174) + N flag (preprocess.cpp:147-193).
void pack_reads(const char* seq, size_t n, int L, uint64_t* packed, uint8_t* has_n);

// a2: stable lexicographic sort of ids + adjacent duplicate links.
void sort_dedupe(const uint64_t* db, int W, std::vector<uint32_t>& ids,
                 uint32_t* next, uint32_t* prev, uint16_t* offset);

// a4 contested runs.  In one overlap pass, suffixes whose [off, L) equals
// the same run of prefixes compete for the run's free prefixes.  In the
// reference each suffix is a thread and a prefix goes to whichever thread's
// atomicCAS (compress.cu:1518) lands first, so the outcome depends on
// scheduling; canonically the suffixes take them in list order.
struct ContestPick {      // in overlap pass `pass`, `suffix` goes before the rest
    int pass;
    uint32_t suffix;
};
struct ContestMember {    // one suffix of a run that two or more suffixes shared
    uint32_t pass;
    uint32_t run;         // index of the run's first prefix in the bucketed prefix list
    uint32_t suffix;
    uint32_t prefix;      // the prefix it took in this pass, or INVALID
};
struct OverlapControl {
    std::vector<ContestPick> picks;        // empty: canonical order
    std::vector<ContestMember>* log = nullptr;
};

// a3+a4: k-mer index over prefix reads and the max_off-1 overlap passes.
// `ctl` (test use only) replays another serialisation of the contested runs
// and records every contested run.  `threads` run the per-pass searches in
// parallel; the links are made in order, so results do not depend on it.
void overlap_link(const Params& p, const uint64_t* db, const std::vector<uint32_t>& sorted_ids,
                  uint32_t* next, uint32_t* prev, uint16_t* offset, const OverlapControl* ctl = nullptr,
                  int threads = 1);

// a5: chain filter; returns (ref ids, unmatched ids), both in sorted order.
void chain_filter(size_t reads_count, const std::vector<uint32_t>& sorted_ids,
                  uint32_t* next, uint32_t* prev, const uint16_t* offset,
                  std::vector<uint32_t>& ref_ids, std::vector<uint32_t>& unmatch_ids);

// a6: exact suffix-prefix merge over every offset on packed reads.
void full_match_packed(const Params& p, const uint64_t* db, std::vector<uint32_t> prefix,
                       std::vector<uint32_t> suffix, uint32_t* next, uint32_t* prev, uint16_t* offset);

// a7: same on ASCII reads (alphabet ACGNT), incl. its own sort + dedupe.
void full_match_ascii(const Params& p, const char* nreads, std::vector<uint32_t> ids, size_t n_total,
                      std::vector<uint32_t>& next, std::vector<uint32_t>& prev, std::vector<uint16_t>& offset);

// a8: chain walk into a pseudogenome.
struct Pseudogenome {
    std::vector<Record> records;
    std::string seq;
};
void assemble_packed(const uint64_t* db, int L, int W, const std::vector<uint32_t>& ids,
                     const uint32_t* next, const uint32_t* prev, const uint16_t* offset,
                     size_t reads_count, Pseudogenome& out);
void assemble_ascii(const char* nreads, int L, const std::vector<uint32_t>& ids,
                    const uint32_t* next, const uint32_t* prev, const uint16_t* offset,
                    size_t reads_count, Pseudogenome& out);
std::vector<uint64_t> pack_ref(const std::string& s);   // compute_binary_ref (+1 pad word)

// a9: map unmatched (packed) and N (ASCII) reads onto the pseudogenome.
struct MapResult {
    std::vector<uint8_t> mm;       // last_mismatch_count per read (U then N)
    std::vector<uint8_t> strand;
    std::vector<uint64_t> pos;
};
void map_reads(const Params& p, const uint64_t* ref, size_t ref_len,
               const uint64_t* udb /*U x W gathered*/, size_t U,
               const char* ndb, size_t NN, MapResult& r, int threads = 1);

// a12: reverse-complement repeat elimination with '%' markers.
struct RefMatcherIndex {
    uint64_t ref_len = 0;
    uint32_t mask = 0;
    std::vector<uint32_t> key_ranges, pos_array;
    const uint64_t* ref = nullptr;
};
void refmatch_index(const uint64_t* ref, uint64_t ref_len, RefMatcherIndex& ix);
// `threads` search the probe groups in parallel; the matches are taken in
// group order, so results do not depend on it.
void refmatch_apply(const RefMatcherIndex& ix, std::string& dest, bool dest_has_n, bool dest_is_ref,
                    std::string& map_off, std::string& map_len, int threads = 1);

// ---- whole block ----
struct BlockInput {
    const uint64_t* db;              // all reads of the block, packed (N as A)
    size_t reads_count;
    std::vector<uint32_t> reads_id;  // non-N ids ascending
    std::vector<char> nreads;        // ASCII of N reads, N_reads_id order
    std::vector<uint32_t> n_ids;     // ids of reads containing N
    std::vector<ContestPick> contest_picks;  // a4 serialisation (empty: canonical)
};

struct BlockStreams {
    uint32_t reads_count = 0;
    char decoder_table[16];                  // ctx A, T, C, G
    std::string ref, unmap_ref, unmap_n_ref; // after '%' compaction
    uint64_t ref_size = 0, unmap_ref_size = 0, unmap_n_ref_size = 0;  // before compaction
    std::string strand;                      // '0'/'1' per record
    std::vector<uint8_t> mis_cnt;
    std::string mis_base;                    // recoded ranks
    std::vector<uint16_t> read_off, unmap_read_off, unmap_n_read_off;  // !PO
    std::vector<uint32_t> pe_order;          // !PO && PE
    std::vector<uint64_t> id_to_pos;         // PO
    std::vector<std::vector<uint16_t>> mis_off;   // [1..max_mismatch]
    std::string ref_off, ref_len_map, unmap_ref_off, unmap_ref_len, unmap_n_ref_off, unmap_n_ref_len;
    // intermediate results exposed for stage-level parity
    std::vector<uint32_t> sorted_ids, next, prev;
    std::vector<uint16_t> offset;
    std::vector<uint32_t> ref_ids, unmatch_ids;
    Pseudogenome hq;
    MapResult map;
    std::vector<Record> records;             // emission order
    std::vector<ContestMember> contests;     // a4 contested runs
};

void compress_block(const Params& p, const BlockInput& in, BlockStreams& out, int threads = 1);

}  // namespace oracle
