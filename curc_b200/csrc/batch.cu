// Batched path: many blocks queued on one context and drained by several
// block pipelines at once (the context's own Block plus extra ones, each
// with its own stream and arena), so that one block's host round trips and
// copies overlap another's kernels.  This replaces the reference's
// one-thread-per-block scheduling (preprocess.cpp:195-242, GPUs taken by a
// mutex spin, compress.cu:52-65) on one device.
#include <algorithm>
#include <atomic>
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

// One block on one worker: reads to the worker's device slot on its stream,
// then the block pipeline.
void run_item(BatchWorker& w, const BatchItem& it) {
    Block& blk = *w.blk;
    const size_t bytes = size_t(it.n) * size_t(it.L);
    const bool pageable = bytes && !is_pinned(it.seqs);
    reserve(w, bytes, pageable);
    const void* src = it.seqs;
    if (pageable) {
        parallel_copy(w.pin, it.seqs, bytes);
        src = w.pin;
    }
    if (bytes) CURC_CHECK(cudaMemcpyAsync(w.dev, src, bytes, cudaMemcpyHostToDevice, blk.stream));
    blk.arena.reset();
    blk.run(w.dev, it.n, it.L, it.po, it.pe);
}

template <class F>
int guarded_batch(curc_ctx* ctx, F&& f) {
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
        for (auto& w : q.pool) w->blk->keep_intermediates = ctx->block->keep_intermediates;
        // every pipeline sized for the largest queued block up front: growing a
        // slot later would allocate (and synchronise) in the middle of the drain
        size_t most = 0;
        bool pageable = false;
        for (const auto& it : items) {
            most = std::max(most, size_t(it.n) * size_t(it.L));
            pageable |= it.n && !curc::is_pinned(it.seqs);
        }
        for (int i = 0; i < W; ++i) curc::reserve(*q.pool[i], most, pageable);
        std::atomic<size_t> next{0};
        std::atomic<bool> stop{false};
        std::mutex cb_mu;
        std::exception_ptr err;
        auto work = [&](curc::BatchWorker& w) {
            try {
                CURC_CHECK(cudaSetDevice(ctx->device));
                for (;;) {
                    if (stop.load()) return;
                    const size_t k = next.fetch_add(1);
                    if (k >= items.size()) return;
                    curc::run_item(w, items[k]);
                    // callbacks one at a time, on this thread, with this block's results
                    std::lock_guard<std::mutex> g(cb_mu);
                    if (stop.load()) return;
                    if (done) {
                        curc::batch_current() = w.blk;
                        const int rc = done(user, items[k].ticket);
                        curc::batch_current() = nullptr;
                        if (rc != 0) throw std::runtime_error("batch drain stopped by the callback");
                    }
                }
            } catch (...) {
                curc::batch_current() = nullptr;
                std::lock_guard<std::mutex> g(cb_mu);
                if (!err) err = std::current_exception();
                stop.store(true);
            }
        };
        std::vector<std::thread> th;
        for (int i = 1; i < W; ++i) th.emplace_back([&, i] { work(*q.pool[i]); });
        work(*q.pool[0]);
        for (auto& t : th) t.join();
        if (err) std::rethrow_exception(err);
        return int(CURC_OK);
    });
}

}  // extern "C"
