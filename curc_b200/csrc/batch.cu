// Batched path: many blocks queued on one context and drained by several
// block pipelines at once (the context's own Block plus extra ones, each
// with its own stream and arena), so that one block's host round trips and
// copies overlap another's kernels.  This replaces the reference's
// one-thread-per-block scheduling (preprocess.cpp:195-242, GPUs taken by a
// mutex spin, compress.cu:52-65) on one device.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <mutex>
#include <stdexcept>
#include <thread>

#include "../../include/curc_b200.h"
#include "block.cuh"

namespace curc {

Block*& batch_current() {
    thread_local Block* b = nullptr;
    return b;
}

BatchWorker::~BatchWorker() {
    if (dev) cudaFree(dev);
    if (pin) cudaFreeHost(pin);
    if (landed) cudaEventDestroy(landed);
}

namespace {

bool is_pinned(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// memcpy with several host threads (pageable -> pinned staging)
void parallel_copy(void* dst, const void* src, size_t bytes) {
    const size_t chunk = size_t(64) << 20;
    const unsigned T = std::max(1u, std::min(8u, unsigned((bytes + chunk - 1) / chunk)));
    if (T == 1) {
        std::memcpy(dst, src, bytes);
        return;
    }
    std::vector<std::thread> th;
    const size_t piece = (bytes + T - 1) / T;
    for (unsigned t = 0; t < T; ++t) {
        const size_t a = std::min(bytes, size_t(t) * piece), b = std::min(bytes, a + piece);
        th.emplace_back([=] { std::memcpy(static_cast<char*>(dst) + a, static_cast<const char*>(src) + a, b - a); });
    }
    for (auto& x : th) x.join();
}

// Input slot (and pinned staging, for pageable input) of at least `bytes`.
void reserve(BatchWorker& w, size_t bytes, bool staging) {
    if (w.dev_cap < bytes + 16) {
        CURC_CHECK(cudaStreamSynchronize(w.blk->stream));
        if (w.dev) CURC_CHECK(cudaFree(w.dev));
        w.dev = nullptr;
        CURC_CHECK(cudaMalloc(&w.dev, bytes + 16));
        w.dev_cap = bytes + 16;
    }
    if (staging && w.pin_cap < bytes) {
        if (w.pin) CURC_CHECK(cudaFreeHost(w.pin));
        w.pin = nullptr;
        CURC_CHECK(cudaHostAlloc(reinterpret_cast<void**>(&w.pin), bytes, cudaHostAllocDefault));
        w.pin_cap = bytes;
    }
}

// Blocks of at least this many bases fill the device on their own: they run
// one at a time from the draining thread, double-buffered over two
// pipelines, instead of on concurrent workers.  (Measured on B200: while one
// worker thread's multi-gigabyte input copy was in flight, the other worker
// thread's block did not start until the copy had landed, so concurrent
// workers hid none of a 3 GB block's 54 ms copy.)
constexpr size_t LARGE_BYTES = size_t(1) << 28;

// CURC_VERBOSE=1: when each block's copy was queued and its run ended.
bool batch_verbose() {
    static const bool v = std::getenv("CURC_VERBOSE") != nullptr;
    return v;
}
double ms_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// Queues the block's reads to the worker's input slot on the queue's copy
// stream (pageable input goes through the worker's pinned staging first).
// The copies have a stream of their own: measured on B200, a 3 GB copy
// queued on one block pipeline's stream held back the kernels of the block
// running on the other pipeline's stream until it had landed, while the same
// copy on a separate stream overlapped them.
void stage_in(BatchQueue& q, BatchWorker& w, const BatchItem& it) {
    const size_t bytes = size_t(it.n) * size_t(it.L);
    const bool pageable = bytes && !is_pinned(it.seqs);
    reserve(w, bytes, pageable);
    if (!w.landed) CURC_CHECK(cudaEventCreateWithFlags(&w.landed, cudaEventDisableTiming));
    const void* src = it.seqs;
    if (pageable) {
        CURC_CHECK(cudaEventSynchronize(w.landed));  // the staging buffer's previous copy
        parallel_copy(w.pin, it.seqs, bytes);
        src = w.pin;
    }
    if (bytes) CURC_CHECK(cudaMemcpyAsync(w.dev, src, bytes, cudaMemcpyHostToDevice, q.copy_stream));
    CURC_CHECK(cudaEventRecord(w.landed, q.copy_stream));
}

// The block pipeline over the worker's input slot, once its copy has landed.
void run_staged(BatchWorker& w, const BatchItem& it, int wi, std::chrono::steady_clock::time_point t0) {
    Block& blk = *w.blk;
    CURC_CHECK(cudaEventSynchronize(w.landed));
    const double tl = batch_verbose() ? ms_since(t0) : 0;
    blk.arena.reset();
    blk.run(w.dev, it.n, it.L, it.po, it.pe);
    if (batch_verbose())
        std::fprintf(stderr, "curc: batch block %u pipeline %d: reads landed %.1f, done %.1f ms (device %.1f)\n",
                     it.ticket, wi, tl, ms_since(t0), blk.stage_ms.count("total") ? blk.stage_ms["total"] : -1.f);
}

template <class F>
int guarded_batch(curc_ctx* ctx, F&& f) {
    if (const int rc = ctx_wait(ctx)) return rc;
    try {
        CURC_CHECK(cudaSetDevice(ctx->device));
        return f();
    } catch (const CudaError& e) {
        ctx->err = e.what();
        return CURC_ERR_CUDA;
    } catch (const std::invalid_argument& e) {
        ctx->err = e.what();
        return CURC_ERR_ARG;
    } catch (const std::exception& e) {
        ctx->err = e.what();
        return CURC_ERR_STATE;
    }
}

}  // namespace
}  // namespace curc

extern "C" {

int curc_batch_submit(curc_ctx* ctx, const char* seqs, uint64_t n, uint16_t read_len, int preserve_order,
                      int paired_end, uint32_t* ticket) {
    if (!ctx || (!seqs && n) || read_len < 1 || read_len > 511) return CURC_ERR_ARG;
    return curc::guarded_batch(ctx, [&] {
        if (!ctx->batch) ctx->batch = std::make_unique<curc::BatchQueue>();
        auto& q = *ctx->batch;
        const uint32_t t = q.next_ticket++;
        q.items.push_back(curc::BatchItem{seqs, n, read_len, preserve_order != 0, paired_end != 0, t});
        if (ticket) *ticket = t;
        return int(CURC_OK);
    });
}

int curc_batch_workers(curc_ctx* ctx, int workers) {
    if (!ctx || workers < 1 || workers > 16) return CURC_ERR_ARG;
    return curc::guarded_batch(ctx, [&] {
        if (!ctx->batch) ctx->batch = std::make_unique<curc::BatchQueue>();
        ctx->batch->workers = workers;
        return int(CURC_OK);
    });
}

int curc_batch_drain(curc_ctx* ctx, curc_block_done_fn done, void* user) {
    if (!ctx) return CURC_ERR_ARG;
    return curc::guarded_batch(ctx, [&] {
        if (!ctx->batch || ctx->batch->items.empty()) return int(CURC_OK);
        auto& q = *ctx->batch;
        std::vector<curc::BatchItem> items;
        items.swap(q.items);
        const int W = int(std::min<size_t>(size_t(q.workers), items.size()));
        while (int(q.pool.size()) < W) {
            auto w = std::make_unique<curc::BatchWorker>();
            if (q.pool.empty()) {
                w->blk = ctx->block.get();
            } else {
                w->own = std::make_unique<curc::Block>();
                w->blk = w->own.get();
            }
            q.pool.push_back(std::move(w));
        }
        for (auto& w : q.pool) {
            w->blk->keep_intermediates = ctx->block->keep_intermediates;
            w->blk->tune = ctx->block->tune;
            w->blk->tune_cache = ctx->block->tune_cache;
        }
        // every pipeline sized for the largest queued block up front: growing a
        // slot later would allocate (and synchronise) in the middle of the drain
        size_t most = 0;
        bool pageable = false;
        for (const auto& it : items) {
            most = std::max(most, size_t(it.n) * size_t(it.L));
            pageable |= it.n && !curc::is_pinned(it.seqs);
        }
        for (int i = 0; i < W; ++i) curc::reserve(*q.pool[i], most, pageable);
        if (!q.copy_stream) CURC_CHECK(cudaStreamCreateWithFlags(&q.copy_stream, cudaStreamNonBlocking));
        std::vector<size_t> large, small;
        for (size_t k = 0; k < items.size(); ++k)
            (size_t(items[k].n) * size_t(items[k].L) >= curc::LARGE_BYTES ? large : small).push_back(k);
        const auto t0 = std::chrono::steady_clock::now();
        auto callback = [&](curc::BatchWorker& w, size_t k) {
            if (!done) return;
            curc::batch_current() = w.blk;
            const int rc = done(user, items[k].ticket);
            curc::batch_current() = nullptr;
            if (rc != 0) throw std::runtime_error("batch drain stopped by the callback");
        };
        // large blocks first, from this thread: while one pipeline runs a
        // block, the next block's reads already cross to the other pipeline's
        // input slot on the copy stream (pageable input is first copied to
        // pinned staging on this thread, which that overlap does not cover)
        if (!large.empty()) {
            const int P = std::min(W, 2);
            try {
                curc::stage_in(q, *q.pool[0], items[large[0]]);
                for (size_t i = 0; i < large.size(); ++i) {
                    curc::BatchWorker& w = *q.pool[i % P];
                    const bool more = i + 1 < large.size();
                    if (more && P > 1) curc::stage_in(q, *q.pool[(i + 1) % P], items[large[i + 1]]);
                    curc::run_staged(w, items[large[i]], int(i % P), t0);
                    callback(w, large[i]);
                    if (more && P == 1) curc::stage_in(q, w, items[large[i + 1]]);
                }
            } catch (...) {
                curc::batch_current() = nullptr;
                // a queued copy may still read the caller's memory: let it land
                if (q.copy_stream) cudaStreamSynchronize(q.copy_stream);
                throw;
            }
        }
        // smaller blocks on concurrent pipelines, one host thread each, so one
        // block's host round trips overlap another's kernels
        std::atomic<size_t> next{0};
        std::atomic<bool> stop{false};
        std::mutex cb_mu;
        std::exception_ptr err;
        auto work = [&](curc::BatchWorker& w, int wi) {
            try {
                CURC_CHECK(cudaSetDevice(ctx->device));
                for (;;) {
                    if (stop.load()) return;
                    const size_t j = next.fetch_add(1);
                    if (j >= small.size()) return;
                    const size_t k = small[j];
                    curc::stage_in(q, w, items[k]);
                    curc::run_staged(w, items[k], wi, t0);
                    // callbacks one at a time, on this thread, with this block's results
                    std::lock_guard<std::mutex> g(cb_mu);
                    if (stop.load()) return;
                    callback(w, k);
                }
            } catch (...) {
                curc::batch_current() = nullptr;
                std::lock_guard<std::mutex> g(cb_mu);
                if (!err) err = std::current_exception();
                stop.store(true);
            }
        };
        if (!small.empty()) {
            const int Ws = int(std::min<size_t>(size_t(W), small.size()));
            std::vector<std::thread> th;
            for (int i = 1; i < Ws; ++i) th.emplace_back([&, i] { work(*q.pool[i], i); });
            work(*q.pool[0], 0);
            for (auto& t : th) t.join();
        }
        // no copy may still read the caller's reads once the drain returns
        if (err) {
            cudaStreamSynchronize(q.copy_stream);
            std::rethrow_exception(err);
        }
        return int(CURC_OK);
    });
}

}  // extern "C"
