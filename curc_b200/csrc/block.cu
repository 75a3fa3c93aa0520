// Block pipeline and C-ABI (include/curc_b200.h).
//
// One block of reads stays resident in HBM from the H2D copy of its ASCII
// sequences to the final streams; only the streams (and, on request, stage
// intermediates for parity checks) come back to the host.
#include <chrono>
#include <future>
#include <cstring>
#include <map>
#include <mutex>
#include <memory>
#include <string>
#include <vector>

#include "../../include/curc_b200.h"
#include "block.cuh"

namespace curc {

namespace {

__global__ void gather_reads_kernel(const uint64_t* __restrict__ db, int W, const uint32_t* __restrict__ ids,
                                    uint32_t m, uint64_t* __restrict__ out) {
    const uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= uint64_t(m) * W) return;
    const uint32_t i = uint32_t(t / W), w = uint32_t(t - uint64_t(i) * W);
    out[t] = db[uint64_t(ids[i]) * W + w];
}

__global__ void ends_kernel(const uint32_t* __restrict__ ids, uint32_t m, const uint32_t* __restrict__ next,
                            const uint32_t* __restrict__ prev, uint8_t* __restrict__ pf, uint8_t* __restrict__ sf) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    pf[i] = prev[ids[i]] == INVALID;
    sf[i] = next[ids[i]] == INVALID;
}

}  // namespace

void Block::run(const uint8_t* d_seq, uint64_t n_reads, int L, bool po, bool pe) {
    if (n_reads > 0xFFFFFFFFull) throw std::runtime_error("more than 2^32-1 reads in one block");
    if (L < 1 || (L + 31) / 32 > 16) throw std::runtime_error("read length must be in [1, 512]");
    p = BlockParams::derive(L, po, pe);
    p.tune = tune;
    if (tune_cache) {
        auto it = tune_cache->find(tune_key(L, n_reads));
        if (it != tune_cache->end()) p.tune = it->second;
    }
    n = uint32_t(n_reads);
    fm_tally = nullptr;
    mo.tally = nullptr;
    host.clear();
    stage_ms.clear();
    pinned.reset();
    StageTimer T{stream, {}, {}};
    struct TimerScope {
        explicit TimerScope(StageTimer* t) { active_timer() = t; }
        ~TimerScope() { active_timer() = nullptr; }
    } timer_scope(&T);
    cudaStream_t s = stream;
    const int W = p.W;
    struct RunEvents {  // released on every exit from the run
        cudaEvent_t a = nullptr, b = nullptr;
        ~RunEvents() {
            if (a) cudaEventDestroy(a);
            if (b) cudaEventDestroy(b);
        }
    } run_ev;
    CURC_CHECK(cudaEventCreate(&run_ev.a));
    CURC_CHECK(cudaEventCreate(&run_ev.b));
    cudaEvent_t ev0 = run_ev.a, ev1 = run_ev.b;
    CURC_CHECK(cudaEventRecord(ev0, s));
    uint32_t* counts = arena.alloc<uint32_t>(16);
    uint32_t* err = arena.alloc<uint32_t>(1);
    CURC_CHECK(cudaMemsetAsync(err, 0, 4, s));

    // a1
    T.begin("pack");
    db = arena.alloc<uint64_t>(size_t(n) * W + 1);
    uint8_t* has_n = arena.alloc<uint8_t>(n ? n : 1);
    {
        SubStage sp("pack.kernel");  // the packing kernel alone (the stage also splits and reads counts back)
        pack_reads(d_seq, n, L, db, has_n, err, s);
    }
    reads_id = arena.alloc<uint32_t>(n ? n : 1);
    n_ids = arena.alloc<uint32_t>(n ? n : 1);
    split_n_reads(has_n, n, reads_id, n_ids, counts, arena, s);
    uint32_t hc[2];
    read_small(hc, counts, 8, s);
    m = hc[0];
    NN = hc[1];
    nreads = arena.alloc<uint8_t>(size_t(NN) * L + 16);
    gather_ascii_rows(d_seq, n_ids, NN, L, nreads, s);
    T.end();
    if (read_scalar(err, s)) throw std::runtime_error("pack: bulk copy wait timed out");
    if (keep_intermediates) {
        keep("packed", db, size_t(n) * W);
        keep("has_n", has_n, n);
    }

    // a2
    T.begin("sort_dedupe");
    next = arena.alloc<uint32_t>(n ? n : 1);
    prev = arena.alloc<uint32_t>(n ? n : 1);
    offset = arena.alloc<uint16_t>(n ? n : 1);
    fill<uint32_t>(next, INVALID, n, s);
    fill<uint32_t>(prev, INVALID, n, s);
    fill<uint16_t>(offset, INVALOFF, n, s);
    sorted = arena.alloc<uint32_t>(m ? m : 1);
    if (m) CURC_CHECK(cudaMemcpyAsync(sorted, reads_id, size_t(m) * 4, cudaMemcpyDeviceToDevice, s));
    {
        SubStage sp("sort_dedupe.radix");
        sort_ids_by_reads(db, W, L, sorted, m, arena, s);
    }
    dedupe_links(db, W, sorted, m, next, prev, offset, s);
    T.end();
    if (keep_intermediates) keep("sorted_ids", sorted, m);

    // a3 + a4
    T.begin("overlap");
    overlap_link(p, db, sorted, m, next, prev, offset, arena, s, &ostats);
    T.end();

    // a5
    T.begin("chain_filter");
    ref_ids = arena.alloc<uint32_t>(m ? m : 1);
    unmatch_ids = arena.alloc<uint32_t>(m ? m : 1);
    chain_filter(n, sorted, m, next, prev, offset, ref_ids, unmatch_ids, counts, arena, s);
    read_small(hc, counts, 8, s);
    n_ref = hc[0];
    U = hc[1];
    T.end();

    // a6 (compress.cu:1576-1591)
    T.begin("full_match");
    fm_tally = arena.alloc<unsigned long long>(3);
    CURC_CHECK(cudaMemsetAsync(fm_tally, 0, 3 * sizeof(unsigned long long), s));
    {
        auto mk = arena.mark();
        uint8_t* pf = arena.alloc<uint8_t>(n_ref ? n_ref : 1);
        uint8_t* sf = arena.alloc<uint8_t>(n_ref ? n_ref : 1);
        uint32_t* pre = arena.alloc<uint32_t>(n_ref ? n_ref : 1);
        uint32_t* suf = arena.alloc<uint32_t>(n_ref ? n_ref : 1);
        if (n_ref) {
            ends_kernel<<<grid_for(n_ref, 256), 256, 0, s>>>(ref_ids, n_ref, next, prev, pf, sf);
            CURC_LAUNCH_CHECK();
        }
        select_flagged(ref_ids, pf, pre, n_ref, counts + 2, arena, s);
        select_flagged(ref_ids, sf, suf, n_ref, counts + 3, arena, s);
        const uint32_t cnt = read_scalar(counts + 3, s);
        full_match_packed(p, db, pre, suf, cnt, next, prev, offset, arena, s, fm_tally);
        arena.release(mk);
    }
    T.end();
    if (keep_intermediates) {
        keep("next", next, n);
        keep("prev", prev, n);
        keep("offset", offset, n);
        keep("ref_ids", ref_ids, n_ref);
        keep("unmatch_ids", unmatch_ids, U);
    }

    // a8
    T.begin("assembly");
    assemble(db, nullptr, L, W, ref_ids, n_ref, n, next, prev, offset, false, hq, arena, s);
    T.end();
    if (keep_intermediates) {
        keep("hq_seq", hq.seq, hq.len);
        keep("hq_records", hq.records, hq.n_records);
    }

    // a9 (compress.cu:1622-1640)
    T.begin("mapping");
    udb = arena.alloc<uint64_t>(size_t(U) * W + 1);
    if (U) {
        gather_reads_kernel<<<grid_for(uint64_t(U) * W, 256), 256, 0, s>>>(db, W, unmatch_ids, U, udb);
        CURC_LAUNCH_CHECK();
    }
    mo.mm = arena.alloc<uint8_t>(U + NN + 1);
    mo.strand = arena.alloc<uint8_t>(U + NN + 1);
    mo.pos = arena.alloc<uint64_t>(U + NN + 1);
    mo.tally = arena.alloc<unsigned long long>(6);
    CURC_CHECK(cudaMemsetAsync(mo.tally, 0, 6 * sizeof(unsigned long long), s));
    map_reads(p, hq.packed, hq.len, udb, U, nreads, NN, mo, arena, s);
    T.end();
    if (keep_intermediates) {
        keep("map_mm", mo.mm, U + NN);
        keep("map_strand", mo.strand, U + NN);
        keep("map_pos", mo.pos, U + NN);
    }

    emit(T);
    CURC_CHECK(cudaEventRecord(ev1, s));
    T.collect(stage_ms);
    CURC_CHECK(cudaStreamSynchronize(s));
    float total = 0;
    CURC_CHECK(cudaEventElapsedTime(&total, ev0, ev1));
    stage_ms["total"] = total;
}

}  // namespace curc

// ---------------------------------------------------------------- C-ABI


namespace curc {
// Error message of the calls that have no context (creation, no-alloc).
std::string& ctxless_error() {
    thread_local std::string e;
    return e;
}

int ctx_wait(curc_ctx* ctx) noexcept {
    if (!ctx->ready.valid()) return CURC_OK;
    // several threads may wait at once (curc -c announces the set-up while
    // it parses); the error text is written under a lock
    static std::mutex err_mu;
    try {
        ctx->ready.get();
    } catch (const std::exception& e) {
        std::lock_guard<std::mutex> g(err_mu);
        ctx->err = e.what();
        return CURC_ERR_CUDA;
    }
    const cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) {
        std::lock_guard<std::mutex> g(err_mu);
        ctx->err = cudaGetErrorString(e);
        return CURC_ERR_CUDA;
    }
    return CURC_OK;
}

bool ctx_ready_now(const curc_ctx* ctx) {
    return !ctx->ready.valid() || ctx->ready.wait_for(std::chrono::seconds(0)) == std::future_status::ready;
}
}  // namespace curc
namespace {

template <class F>
int guarded(curc_ctx* ctx, F&& f) {
    if (ctx)
        if (const int rc = curc::ctx_wait(ctx)) return rc;
    try {
        if (ctx) CURC_CHECK(cudaSetDevice(ctx->device));
        f();
        return CURC_OK;
    } catch (const curc::CudaError& e) {
        if (ctx) ctx->err = e.what();
        return CURC_ERR_CUDA;
    } catch (const std::invalid_argument& e) {
        if (ctx) ctx->err = e.what();
        return CURC_ERR_ARG;
    } catch (const std::exception& e) {
        if (ctx) ctx->err = e.what();
        return CURC_ERR_STATE;
    }
}
}  // namespace

extern "C" {

int curc_ctx_create(int device, curc_ctx** out) {
    if (!out) return CURC_ERR_ARG;
    *out = nullptr;
    try {
        int count = 0;
        CURC_CHECK(cudaGetDeviceCount(&count));
        if (device < 0 || device >= count) throw std::invalid_argument("no such CUDA device");
        CURC_CHECK(cudaSetDevice(device));
        auto* c = new curc_ctx;
        c->device = device;
        c->block = std::make_unique<curc::Block>();
        *out = c;
        return CURC_OK;
    } catch (const std::exception& e) {
        curc::ctxless_error() = e.what();
        return CURC_ERR_CUDA;
    }
}

int curc_device_count(int* count) {
    if (!count) return CURC_ERR_ARG;
    *count = 0;
    const cudaError_t e = cudaGetDeviceCount(count);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *count = 0;
        curc::ctxless_error() = cudaGetErrorString(e);
        return CURC_ERR_CUDA;
    }
    return CURC_OK;
}

int curc_ctx_create_deferred(int device, curc_ctx** out) {
    if (!out) return CURC_ERR_ARG;
    *out = nullptr;
    try {
        auto* c = new curc_ctx;
        c->device = device;
        // driver start, primary context and the pipeline's stream, on a
        // thread of their own; the calls that need them wait (ctx_wait)
        c->ready = std::async(std::launch::async, [c, device] {
                       int count = 0;
                       CURC_CHECK(cudaGetDeviceCount(&count));
                       if (device < 0 || device >= count) throw std::invalid_argument("no such CUDA device");
                       CURC_CHECK(cudaSetDevice(device));
                       CURC_CHECK(cudaFree(nullptr));
                       c->block = std::make_unique<curc::Block>();
                   }).share();
        *out = c;
        return CURC_OK;
    } catch (const std::exception& e) {
        curc::ctxless_error() = e.what();
        return CURC_ERR_STATE;
    }
}

int curc_ctx_wait(curc_ctx* ctx) {
    if (!ctx) return CURC_ERR_ARG;
    return curc::ctx_wait(ctx);
}

void curc_ctx_destroy(curc_ctx* ctx) {
    if (!ctx) return;
    if (ctx->ready.valid()) ctx->ready.wait();
    cudaSetDevice(ctx->device);
    delete ctx;
}

const char* curc_last_error(const curc_ctx* ctx) { return ctx ? ctx->err.c_str() : curc::ctxless_error().c_str(); }

int curc_pack_device(curc_ctx* ctx, const char* seqs_dev, uint64_t n, uint16_t read_len, uint64_t* packed_dev,
                     uint8_t* has_n_dev, void* stream) {
    if (!ctx || (!seqs_dev && n) || (!packed_dev && n) || (!has_n_dev && n)) return CURC_ERR_ARG;
    if (ctx)
        if (const int rc = curc::ctx_wait(ctx)) return rc;
    if (read_len < 1 || read_len > 512) {
        ctx->err = "read length must be in [1, 512]";
        return CURC_ERR_ARG;
    }
    return guarded(ctx, [&] {
        cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->block->stream;
        curc::Arena& a = ctx->block->arena;
        auto mk = a.mark();
        uint32_t* err = a.alloc<uint32_t>(1);
        CURC_CHECK(cudaMemsetAsync(err, 0, 4, s));
        curc::pack_reads(reinterpret_cast<const uint8_t*>(seqs_dev), n, read_len, packed_dev, has_n_dev, err, s);
        const uint32_t e = curc::read_scalar(err, s);
        a.release(mk);
        if (e) throw std::runtime_error("pack: bulk copy wait timed out");
    });
}

int curc_block_run_device(curc_ctx* ctx, const char* seqs_dev, uint64_t n, uint16_t read_len, int preserve_order,
                          int paired_end) {
    if (!ctx || (!seqs_dev && n)) return CURC_ERR_ARG;
    if (ctx)
        if (const int rc = curc::ctx_wait(ctx)) return rc;
    return guarded(ctx, [&] {
        ctx->block->arena.reset();
        ctx->block->run(reinterpret_cast<const uint8_t*>(seqs_dev), n, read_len, preserve_order != 0,
                        paired_end != 0);
    });
}

int curc_block_run(curc_ctx* ctx, const char* seqs, uint64_t n, uint16_t read_len, int preserve_order,
                   int paired_end) {
    if (!ctx || (!seqs && n)) return CURC_ERR_ARG;
    if (ctx)
        if (const int rc = curc::ctx_wait(ctx)) return rc;
    return guarded(ctx, [&] {
        curc::Block& b = *ctx->block;
        b.arena.reset();
        const size_t bytes = size_t(n) * read_len;
        uint8_t* d = b.arena.alloc<uint8_t>(bytes + 16);
        CURC_CHECK(cudaMemcpyAsync(d, seqs, bytes, cudaMemcpyHostToDevice, b.stream));
        b.run(d, n, read_len, preserve_order != 0, paired_end != 0);
    });
}

int curc_block_get(curc_ctx* ctx, const char* name, const void** ptr, uint64_t* bytes) {
    if (!ctx || !name || !ptr || !bytes) return CURC_ERR_ARG;
    if (ctx)
        if (const int rc = curc::ctx_wait(ctx)) return rc;
    const curc::Block* blk = curc::batch_current() ? curc::batch_current() : ctx->block.get();
    auto it = blk->host.find(name);
    if (it == blk->host.end()) {
        ctx->err = std::string("unknown result: ") + name;
        return CURC_ERR_ARG;
    }
    *ptr = it->second.ptr;
    *bytes = it->second.size;
    return CURC_OK;
}

int curc_ctx_trim(curc_ctx* ctx) {
    if (!ctx) return CURC_ERR_ARG;
    if (ctx)
        if (const int rc = curc::ctx_wait(ctx)) return rc;
    if (ctx->batch && !ctx->batch->items.empty()) {
        ctx->err = "trim: blocks are queued for a drain";
        return CURC_ERR_STATE;
    }
    return guarded(ctx, [&] {
        CURC_CHECK(cudaStreamSynchronize(ctx->block->stream));
        if (ctx->batch) ctx->batch->pool.clear();  // the extra pipelines, input slots and staging
        ctx->block->arena.trim();
    });
}

int curc_ctx_keep_intermediates(curc_ctx* ctx, int keep) {
    if (!ctx) return CURC_ERR_ARG;
    if (ctx)
        if (const int rc = curc::ctx_wait(ctx)) return rc;
    ctx->block->keep_intermediates = keep != 0;
    return CURC_OK;
}

uint64_t curc_kernel_launches(void) { return curc::launches(); }

int curc_block_stage_ms(curc_ctx* ctx, const char* stage, float* ms) {
    if (!ctx || !stage || !ms) return CURC_ERR_ARG;
    if (ctx)
        if (const int rc = curc::ctx_wait(ctx)) return rc;
    auto it = ctx->block->stage_ms.find(stage);
    if (it == ctx->block->stage_ms.end()) {
        ctx->err = std::string("unknown stage: ") + stage;
        return CURC_ERR_ARG;
    }
    *ms = it->second;
    return CURC_OK;
}

}  // extern "C"
