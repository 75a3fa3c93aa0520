// Host side of the drop-in `curc -c`: FASTQ ingest with the reference's
// block split, block stream coding, archive layout.  No CUDA types here.
#pragma once
#include <cstdint>
#include <functional>
#include <map>
#include <string>
#include <vector>

namespace curc {
namespace host {

struct Buf {
    const uint8_t* ptr = nullptr;
    size_t size = 0;
};

// The streams of one compressed block, by the names of curc_block_get.
struct BlockView {
    uint32_t reads_count = 0;
    int read_len = 0;
    bool preserve_order = false, paired_end = false;
    std::map<std::string, Buf> streams;
    const Buf& get(const char* name) const;
    // learned mismatch coding (learned mode only): the serialised model and
    // the block's learned stream; empty in plain mode
    std::string learned_model, learned_stream;
};

// Coder byte of the mismatch-base container when the block's mismatch bases
// and offsets are coded by the learned coder (the container's other coder
// bytes are LzmaLib.h's LZMA_CODER 1, PPMD7_CODER 3, VARLEN_DNA_CODER 11).
constexpr uint8_t LEARNED_CODER = 100;

struct CoderParams {
    int flzma2_level = 10;    // --flzma2_level
    int flzma2_threads = 16;  // --flzma2_thread_num
    std::string bsc_path;     // the bsc executable (strand stream)
    std::string tmpdir;       // scratch files for bsc
    // called (from coder threads) with each coder's name and seconds
    std::function<void(const char*, double)> on_time;
    // learned mode: called with the bytes of the plain and of the learned
    // coding of a block's mismatch bases and offsets
    std::function<void(uint64_t, uint64_t)> on_learned;
};

// Block body in the reference layout (compress.cu:1364-2146).
std::string encode_block(const BlockView& v, const CoderParams& cp);
// Coded sizes of a block's mismatch streams with the plain coders (the
// same calls as encode_block): counts, bases, offsets.
void plain_mismatch_bytes(const BlockView& v, uint64_t out[3]);
// Sizes of the same raw mismatch streams (counts, bases, offsets) under the
// general-purpose coders of the block's other streams: fast-lzma2 at the
// configured level and libbsc (for comparison with the learned coder).
void general_mismatch_bytes(const BlockView& v, const CoderParams& cp, uint64_t out[2]);
// Archive header (preprocess.cpp:261-266).
std::string archive_header(bool po, bool pe, int read_len, int blocks);

// The learned mismatch stream of a block decoded (learned::decode_stream)
// by this host-compiled translation unit, whose copy of the host network
// runs on the CPU's byte dot products where it has them; the arguments are
// decode_stream's, with the model as its serialised bytes (sizeof(Model)).
std::string learned_decode(const void* model, const uint8_t* p, size_t bytes, const uint8_t* ref, uint64_t rl, int L,
                           size_t records, const uint64_t* pos, const uint8_t* strand, const uint8_t* cnt,
                           uint16_t* off, char* base);

// FASTQ ingest.  Reads single-end (f2 empty) or paired-end files in the
// reference's 50 MB windows (25 MB per mate) cut at record boundaries by its
// header heuristic, and closes a block once the bytes read since the last
// cut exceed block_ratio of the input (preprocess.cpp:66-254).  The
// sequences go to the sink window by window, n x L ASCII bytes in block
// order (mates interleaved).
struct IngestSink {
    virtual ~IngestSink() = default;
    // a block starts; its sequences take at most max_bytes
    virtual void begin_block(size_t max_bytes, int L) = 0;
    // where the next window's sequences go (at most `bytes`)
    virtual char* window_buffer(size_t bytes) = 0;
    // the window's `reads` sequences are in the buffer
    virtual void window_done(uint64_t reads) = 0;
    virtual void end_block() = 0;
};
struct IngestResult {
    int read_len = 0;
    uint64_t reads = 0;
    int blocks = 0;
};
IngestResult ingest_fastq(const std::string& f1, const std::string& f2, double block_ratio, IngestSink& sink);

// Product decoder: a `.curc` archive to <out_prefix>.seq (single-end) or
// <out_prefix>_1.seq and _2.seq (paired-end), one read per line, in the
// reference decoder's order (decompress.cu:760-1060).  Host only.
struct DecodeParams {
    std::string bsc_path;  // the bsc executable (strand stream)
    std::string tmpdir;    // scratch files for bsc
    int threads = 0;       // host threads (0: all)
};
struct DecodeResult {
    uint64_t reads = 0;
    int blocks = 0, read_len = 0;
    bool paired_end = false, preserve_order = false;
};
DecodeResult decode_archive(const std::string& archive, const std::string& out_prefix, const DecodeParams& p);
// Layout of an archive without decoding it: flags, read length, and each
// block's body size and read count.
struct ArchiveInfo {
    bool preserve_order = false, paired_end = false;
    int read_len = 0;
    std::vector<uint64_t> block_bytes;
    std::vector<uint32_t> block_reads;
};
ArchiveInfo archive_info(const std::string& archive);

// Read length of the first record (preprocess.cpp:286-300).
int first_read_length(const std::string& f1);

}  // namespace host
}  // namespace curc
