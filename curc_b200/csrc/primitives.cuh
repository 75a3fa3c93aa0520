// Device-wide primitives used by every stage: a bump arena over device
// memory, exclusive scan, stable compaction, and a stable LSD radix sort.
// All are deterministic: results never depend on thread scheduling.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include "common.cuh"

namespace curc {

uint64_t launches();

// Bump allocator over large device chunks.  reset() keeps the memory, so a
// pipeline that runs block after block allocates device memory only while
// it grows; when a run needed more than one chunk, reset() replaces them by
// one chunk of the largest run's size.  Alignment 256 bytes (TMA and vector
// loads need 16).
class Arena {
public:
    explicit Arena(size_t chunk = size_t(1) << 30) : chunk_(chunk) {}
    ~Arena();
    Arena(const Arena&) = delete;
    Arena& operator=(const Arena&) = delete;

    void* alloc_bytes(size_t bytes);
    template <class T>
    T* alloc(size_t n) { return static_cast<T*>(alloc_bytes(n * sizeof(T))); }
    void reset();
    // Frees every chunk (nothing may be in use: the stream work that used
    // them must have completed; cudaFree waits for the device).
    void trim();
    size_t high_water() const { return high_water_; }
    size_t in_use() const;

    // Marks let a stage release its scratch once it is done.
    struct Mark { size_t chunk, used; };
    Mark mark() const { return {cur_, cur_ < chunks_.size() ? chunks_[cur_].used : 0}; }
    void release(const Mark& m);

private:
    struct Chunk { char* base; size_t size, used; };
    std::vector<Chunk> chunks_;
    size_t cur_ = 0;
    size_t chunk_;
    size_t high_water_ = 0;
};

// Growable pinned host memory, bump allocated, reset per block; results are
// copied into it asynchronously and returned as views.
class PinnedArena {
public:
    PinnedArena() = default;
    ~PinnedArena();
    PinnedArena(const PinnedArena&) = delete;
    PinnedArena& operator=(const PinnedArena&) = delete;
    // moving hands the chunks over (views into them stay valid)
    PinnedArena(PinnedArena&& o) noexcept : chunks_(std::move(o.chunks_)), cur_(o.cur_) {
        o.chunks_.clear();
        o.cur_ = 0;
    }
    PinnedArena& operator=(PinnedArena&& o) noexcept;
    uint8_t* alloc(size_t bytes);
    void reset();

private:
    struct Chunk { uint8_t* base; size_t size, used; };
    std::vector<Chunk> chunks_;
    size_t cur_ = 0;
};

// CUDA events around the stages of one block run (nested names allowed,
// e.g. "refmatch" and "refmatch.probe"); collect() adds each span's time.
struct StageTimer {
    cudaStream_t s;
    struct Span { std::string name; cudaEvent_t a, b; };
    std::vector<Span> ev;
    std::vector<size_t> open;
    size_t begin_span(const std::string& name);
    void end_span(size_t i);
    void begin(const std::string& name) { open.push_back(begin_span(name)); }
    void end() {
        end_span(open.back());
        open.pop_back();
    }
    void collect(std::map<std::string, float>& out);
    // spans not collected (a run that threw) release their events here
    ~StageTimer() {
        for (auto& e : ev) {
            cudaEventDestroy(e.a);
            cudaEventDestroy(e.b);
        }
    }
};

// The timer of the block run in progress on this thread (or null).
StageTimer*& active_timer();

// Times a scope as a sub-stage of the running block, if any.
struct SubStage {
    StageTimer* t;
    size_t i = 0;
    // on = false: no span (launches being captured into a graph)
    explicit SubStage(const char* name, bool on = true) : t(on ? active_timer() : nullptr) {
        if (t) i = t->begin_span(name);
    }
    void stop() {
        if (t) t->end_span(i);
        t = nullptr;
    }
    ~SubStage() { stop(); }
};

// out[i] = sum(in[0..i)); optionally *total = sum(in[0..n)) (device pointer).
// In-place (out == in) is allowed.
template <class T>
void exclusive_scan(const T* in, T* out, size_t n, T* total, Arena& a, cudaStream_t s);

// Stable compaction: out = [in[i] for i if flags[i]], *count = number kept.
template <class T>
void select_flagged(const T* in, const uint8_t* flags, T* out, size_t n, uint32_t* count, Arena& a,
                    cudaStream_t s);

// Same, writing the indices i with flags[i] set.
void select_indices(const uint8_t* flags, uint32_t* out, size_t n, uint32_t* count, Arena& a, cudaStream_t s);

// Stable LSD radix sort of (key, value) pairs on key bits [begin_bit,
// end_bit).  keys/vals are overwritten with the sorted sequence.  vals may be
// null (keys only).
template <class K, class V>
void radix_sort_pairs(K* keys, V* vals, size_t n, int begin_bit, int end_bit, Arena& a, cudaStream_t s);

// Stable sort of ids by packed read content (W words per read, lexicographic
// over all words): ids is permuted in place.
void sort_ids_by_reads(const uint64_t* db, int W, int L, uint32_t* ids, size_t n, Arena& a, cudaStream_t s);

// Gather 64-bit words: out[i] = src[idx[i] * stride + word].
void gather_words(const uint64_t* src, const uint32_t* idx, size_t n, int stride, int word, uint64_t* out,
                  cudaStream_t s);

template <class T>
void fill(T* p, T v, size_t n, cudaStream_t s);

void iota(uint32_t* p, size_t n, cudaStream_t s);

// Reads back `bytes` (at most 4 KiB) of device memory after the stream's
// work so far, and synchronises the stream.  A one-block kernel stores them
// into mapped pinned host memory (one buffer per host thread), so the read
// never waits on a copy engine: another pipeline's multi-gigabyte input copy
// on the same device cannot hold it back.
void read_small(void* host, const void* dev, size_t bytes, cudaStream_t s);

// Reads back one device value (synchronises the stream).
template <class T>
T read_scalar(const T* dev, cudaStream_t s) {
    T v;
    read_small(&v, dev, sizeof(T), s);
    return v;
}

}  // namespace curc
