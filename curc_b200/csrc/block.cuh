// Device-resident state of one block and the pipeline driver.
#pragma once
#include <future>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "learned_model.hpp"
#include "stages.cuh"

namespace curc {

// A result returned to the host: a view into pinned staging memory (filled
// by an async copy on the block's stream) or an owned small vector.
struct HostBuf {
    const uint8_t* ptr = nullptr;
    size_t size = 0;
    std::vector<uint8_t> own;
};

struct Block {
    cudaStream_t stream = nullptr;
    Arena arena;
    bool keep_intermediates = true;
    Tuning tune;  // launch and table choices for the next runs (no effect on results)
    // when set: per-block choices by (read length, read-count bucket); blocks
    // whose bucket is missing use `tune`
    std::shared_ptr<const std::map<TuneKey, Tuning>> tune_cache;

    BlockParams p;
    uint32_t n = 0, m = 0, NN = 0, n_ref = 0, U = 0;
    uint64_t* db = nullptr;
    uint32_t *reads_id = nullptr, *n_ids = nullptr, *sorted = nullptr, *next = nullptr, *prev = nullptr;
    uint32_t *ref_ids = nullptr, *unmatch_ids = nullptr;
    uint16_t* offset = nullptr;
    uint8_t* nreads = nullptr;
    uint64_t* udb = nullptr;
    Assembled hq;
    MapOut mo;
    OverlapStats ostats;
    unsigned long long* fm_tally = nullptr;  // full-match counters (device, 3)
    // emission
    uint32_t n_map = 0, n_records = 0, n_ug = 0, n_un = 0, n_mis = 0;
    uint32_t *ug = nullptr, *un = nullptr, *pe_order = nullptr;
    uint64_t* id_to_pos = nullptr;
    DevRecord* srec = nullptr;
    uint8_t *smis = nullptr, *mctx = nullptr, *mbase = nullptr;
    std::vector<uint32_t> class_count;
    uint64_t class_elems = 0;
    uint16_t* off_all = nullptr;
    Assembled lq, lqn;

    std::map<std::string, HostBuf> host;
    PinnedArena pinned;
    std::map<std::string, float> stage_ms;

    Block() { CURC_CHECK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking)); }
    ~Block() {
        if (stream) cudaStreamDestroy(stream);
    }
    Block(const Block&) = delete;
    Block& operator=(const Block&) = delete;

    void run(const uint8_t* d_seq, uint64_t n_reads, int L, bool po, bool pe);
    // a10-a12: stream emission, unmapped pseudogenomes, repeat removal
    void emit(StageTimer& T);
    // a12 on the three pseudogenomes; fills the ref / map streams
    void refmatch_all();

    // D2H copy of a device array into pinned staging (async on the stream)
    template <class T>
    void keep(const std::string& name, const T* dev, size_t count) {
        HostBuf b;
        b.size = count * sizeof(T);
        if (count) {
            uint8_t* p = pinned.alloc(b.size);
            CURC_CHECK(cudaMemcpyAsync(p, dev, b.size, cudaMemcpyDeviceToHost, stream));
            b.ptr = p;
        }
        host[name] = std::move(b);
    }
    void put(const std::string& name, std::vector<uint8_t>&& v) {
        HostBuf b;
        b.own = std::move(v);
        b.ptr = b.own.data();
        b.size = b.own.size();
        host[name] = std::move(b);
    }
};

}  // namespace curc

namespace curc {

// Blocks queued for curc_batch_drain: the caller's host reads (valid until
// the drain returns).  The drain runs them on several block pipelines at
// once (each a Block with its own stream, arena and input slot), so one
// block's copies and host round trips overlap another's kernels.
struct BatchItem {
    const char* seqs;
    uint64_t n;
    int L;
    bool po, pe;
    uint32_t ticket;
};
struct BatchWorker {
    Block* blk = nullptr;               // the context's own block, or `own`
    std::unique_ptr<Block> own;
    uint8_t* dev = nullptr;             // device input slot
    size_t dev_cap = 0;
    uint8_t* pin = nullptr;             // pinned staging for pageable input
    size_t pin_cap = 0;
    cudaEvent_t landed = nullptr;       // the last copy into `dev` has completed
    ~BatchWorker();
};
struct BatchQueue {
    std::vector<BatchItem> items;
    uint32_t next_ticket = 0;
    int workers = 2;
    std::vector<std::unique_ptr<BatchWorker>> pool;
    cudaStream_t copy_stream = nullptr;  // every input copy of the drains
    ~BatchQueue() {
        if (copy_stream) cudaStreamDestroy(copy_stream);
    }
};

// The block whose results curc_block_get returns on this thread while a
// drain callback runs (null otherwise).
Block*& batch_current();

namespace learned {
// The learned mismatch stream of a block's last run (learned.cu).
std::string encode_stream(const Model& model, Block& b);
}  // namespace learned

}  // namespace curc

// The C-ABI context (include/curc_b200.h): one device, one block pipeline.
struct curc_ctx {
    int device = 0;
    std::unique_ptr<curc::Block> block;
    std::unique_ptr<curc::BatchQueue> batch;
    // set: whole-file compression also tries the learned mismatch coder
    std::unique_ptr<curc::learned::Model> mismatch_model;
    std::string err;
    // curc_ctx_create_deferred: the CUDA set-up running on its own thread
    // (`block` exists once it is ready); invalid for curc_ctx_create
    std::shared_future<void> ready;
    curc_ctx() = default;
    curc_ctx(const curc_ctx&) = delete;
    curc_ctx& operator=(const curc_ctx&) = delete;
    ~curc_ctx() {
        if (ready.valid()) ready.wait();
    }
};

namespace curc {
// Waits for a deferred context's CUDA set-up (then makes its device current
// on the calling thread): CURC_OK, or the set-up's error (in ctx->err).
int ctx_wait(curc_ctx* ctx) noexcept;
// Whether the set-up of a deferred context has finished (always true for
// a context made by curc_ctx_create).
bool ctx_ready_now(const curc_ctx* ctx);
}  // namespace curc
