// Whole-file compression through the device path: FASTQ ingest, one block
// run per block, stream coding on host threads overlapped with the next
// block's ingest and device work, archive in the reference layout
// (the reference's process() + block_compress(), preprocess.cpp:66-283).
#include <unistd.h>

#include <chrono>
#include <cstring>
#include <cstdio>
#include <cstdlib>
#include <future>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/curc_b200.h"
#include "block.cuh"
#include "host/host.hpp"


namespace curc {

namespace {

// A block's streams, owned for the coder threads: the block's pinned arena
// (the streams copied back from the device) and its host-made streams are
// handed over, not copied, and the block starts its next run with a fresh
// arena.  The block keeps no views of them.
struct Snapshot {
    host::BlockView view;
    PinnedArena pinned;
    std::vector<std::vector<uint8_t>> store;
};

std::shared_ptr<Snapshot> snapshot(Block& b) {
    auto s = std::make_shared<Snapshot>();
    s->view.reads_count = b.n;
    s->view.read_len = b.p.L;
    s->view.preserve_order = b.p.preserve_order;
    s->view.paired_end = b.p.paired_end;
    s->pinned = std::move(b.pinned);
    s->store.reserve(b.host.size());
    for (auto& kv : b.host) {
        if (!kv.second.own.empty()) {
            s->store.push_back(std::move(kv.second.own));
            s->view.streams[kv.first] = host::Buf{s->store.back().data(), s->store.back().size()};
        } else {
            s->view.streams[kv.first] = host::Buf{kv.second.ptr, kv.second.size};
        }
    }
    b.host.clear();
    return s;
}

// Ingest sink that streams each window's sequences to the device: parsed
// into one of two pinned staging buffers, copied asynchronously into the
// block's device input while the next window is read and parsed; the block
// then runs and its streams are coded on a host thread.
// Host-stage seconds of one whole-file run, summed over its blocks (coder
// threads add theirs concurrently).
struct FileTimes {
    std::mutex mu;
    double ingest = 0, device = 0, snapshot = 0, coders = 0;
    uint64_t mis_plain = 0, mis_learned = 0, learned_blocks = 0;  // learned mode: mismatch bytes per coding
    std::map<std::string, double> coder;
    void add_coder(const char* what, double s) {
        std::lock_guard<std::mutex> g(mu);
        coder[what] += s;
    }
};

// With a deferred context (curc_ctx_create_deferred) the sink does not wait
// for CUDA: until the context is ready, windows are parsed into host
// buffers of their own, and once it is (looked at every window, waited for
// at the block's end) they are copied to the device in order and the sink
// continues as above.  The set-up thus runs while the FASTQ files are read.
class DeviceSink : public host::IngestSink {
public:
    DeviceSink(curc_ctx* ctx, bool po, bool pe, const host::CoderParams& cp, bool verbose, FileTimes& times,
               const learned::Model* model)
        : ctx_(ctx), po_(po), pe_(pe), cp_(cp), verbose_(verbose), times_(times), model_(model) {
        cp_.on_time = [t = &times_](const char* what, double s) { t->add_coder(what, s); };
        cp_.on_learned = [t = &times_](uint64_t plain, uint64_t learned) {
            std::lock_guard<std::mutex> g(t->mu);
            t->mis_plain += plain;
            t->mis_learned += learned;
            t->learned_blocks += learned < plain;
        };
    }
    ~DeviceSink() override {
        if (!blk_) return;
        for (auto& e : ev_) cudaEventSynchronize(e);
        for (auto& e : ev_) cudaEventDestroy(e);
        for (auto& b : stage_)
            if (b.ptr) cudaFreeHost(b.ptr);
        blk_->keep_intermediates = keep_inter_;
    }
    // The context's block, once CUDA is ready (wait: block until it is).
    bool attach(bool wait) {
        if (blk_) return true;
        if (!wait && !ctx_ready_now(ctx_)) return false;
        if (ctx_wait(ctx_) != CURC_OK) throw CudaError(cudaErrorInitializationError, ctx_->err.c_str());
        Block* b = ctx_->block.get();
        for (auto& e : ev_) CURC_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        keep_inter_ = b->keep_intermediates;
        b->keep_intermediates = false;
        blk_ = b;
        return true;
    }
    void begin_block(size_t max_bytes, int L) override {
        t_begin_ = clk::now();
        L_ = L;
        max_bytes_ = max_bytes;
        reads_ = 0;
        dev_open_ = false;
        if (attach(false)) open_device_block();
    }
    char* window_buffer(size_t bytes) override {
        if (!attach(false)) {
            host_win_ = true;
            pend_.push_back(Pending{std::unique_ptr<char[]>(new char[bytes]), 0});
            return pend_.back().data.get();
        }
        host_win_ = false;
        flush_pending();
        cur_ ^= 1;
        Stage& st = stage_[cur_];
        CURC_CHECK(cudaEventSynchronize(ev_[cur_]));  // its last copy is done
        if (st.size < bytes) {
            if (st.ptr) CURC_CHECK(cudaFreeHost(st.ptr));
            st.ptr = nullptr;
            CURC_CHECK(cudaHostAlloc(reinterpret_cast<void**>(&st.ptr), bytes, cudaHostAllocDefault));
            st.size = bytes;
        }
        return st.ptr;
    }
    void window_done(uint64_t reads) override {
        const size_t bytes = size_t(reads) * size_t(L_);
        reads_ += reads;
        if (host_win_) {
            pend_.back().bytes = bytes;
            return;
        }
        if (off_ + bytes > cap_) throw std::runtime_error("ingest: block larger than its bound");
        if (bytes)
            CURC_CHECK(cudaMemcpyAsync(dev_ + off_, stage_[cur_].ptr, bytes, cudaMemcpyHostToDevice, blk_->stream));
        CURC_CHECK(cudaEventRecord(ev_[cur_], blk_->stream));
        off_ += bytes;
    }
    void end_block() override {
        attach(true);
        flush_pending();
        const auto ta = clk::now();
        blk_->run(dev_, reads_, L_, po_, pe_);
        const auto tb = clk::now();
        auto snap = snapshot(*blk_);
        if (model_) {
            // learned mode: the block's learned mismatch stream, from the
            // block's device state before the next block reuses it; the
            // writer keeps it when it is smaller than the plain coding
            const auto l0 = clk::now();
            snap->view.learned_stream = learned::encode_stream(*model_, *blk_);
            snap->view.learned_model.assign(reinterpret_cast<const char*>(model_), sizeof(learned::Model));
            times_.add_coder("learned", secs(l0, clk::now()));
        }
        const auto tc = clk::now();
        const size_t bi = bodies.size();
        const bool verbose = verbose_;
        const host::CoderParams cp = cp_;
        FileTimes* times = &times_;
        {
            std::lock_guard<std::mutex> g(times_.mu);
            times_.ingest += secs(t_begin_, ta);
            times_.device += secs(ta, tb);
            times_.snapshot += secs(tb, tc);
        }
        bodies.push_back(std::async(std::launch::async, [snap, cp, verbose, bi, times] {
            const auto e0 = clk::now();
            std::string body = host::encode_block(snap->view, cp);
            const double s = secs(e0, clk::now());
            {
                std::lock_guard<std::mutex> g(times->mu);
                times->coders += s;
            }
            if (verbose) std::fprintf(stderr, "curc: block %zu coders %.3f s\n", bi, s);
            return body;
        }));
        if (verbose_)
            std::fprintf(stderr, "curc: block %zu ingest and copy %.3f s, device %.3f s, snapshot %.3f s (%llu reads)\n",
                         bi, secs(t_begin_, ta), secs(ta, tb), secs(tb, tc), (unsigned long long)reads_);
    }
    std::vector<std::future<std::string>> bodies;

private:
    using clk = std::chrono::steady_clock;
    static double secs(clk::time_point a, clk::time_point b) { return std::chrono::duration<double>(b - a).count(); }
    struct Stage {
        char* ptr = nullptr;
        size_t size = 0;
    };
    // the device side of the current block: its input in the arena
    void open_device_block() {
        blk_->arena.reset();
        dev_ = blk_->arena.alloc<uint8_t>(max_bytes_ + 16);
        cap_ = max_bytes_;
        off_ = 0;
        dev_open_ = true;
    }
    // windows parsed before the context was ready, copied in order
    void flush_pending() {
        if (!dev_open_) open_device_block();
        if (pend_.empty()) return;
        for (auto& w : pend_) {
            if (off_ + w.bytes > cap_) throw std::runtime_error("ingest: block larger than its bound");
            // pageable source: the call returns once the bytes are staged
            if (w.bytes) CURC_CHECK(cudaMemcpyAsync(dev_ + off_, w.data.get(), w.bytes, cudaMemcpyHostToDevice,
                                                    blk_->stream));
            off_ += w.bytes;
        }
        CURC_CHECK(cudaStreamSynchronize(blk_->stream));
        pend_.clear();
    }
    struct Pending {
        std::unique_ptr<char[]> data;
        size_t bytes;
    };
    curc_ctx* ctx_;
    Block* blk_ = nullptr;
    bool keep_inter_ = false;
    std::vector<Pending> pend_;
    bool host_win_ = false, dev_open_ = false;
    size_t max_bytes_ = 0;
    bool po_, pe_;
    host::CoderParams cp_;
    bool verbose_;
    FileTimes& times_;
    const learned::Model* model_;
    Stage stage_[2];
    cudaEvent_t ev_[2] = {nullptr, nullptr};
    int cur_ = 0, L_ = 0;
    uint8_t* dev_ = nullptr;
    size_t cap_ = 0, off_ = 0;
    uint64_t reads_ = 0;
    clk::time_point t_begin_;
};

}  // namespace

}  // namespace curc

namespace curc {
namespace host {
const Buf& BlockView::get(const char* name) const {
    auto it = streams.find(name);
    if (it == streams.end()) throw std::runtime_error(std::string("missing stream ") + name);
    return it->second;
}
}  // namespace host
}  // namespace curc

extern "C" int curc_ctx_set_mismatch_model(curc_ctx* ctx, const void* model, uint64_t bytes) {
    if (!ctx) return CURC_ERR_ARG;
    if (!model || !bytes) {
        ctx->mismatch_model.reset();
        return CURC_OK;
    }
    if (bytes != sizeof(curc::learned::Model)) {
        ctx->err = "mismatch model: " + std::to_string(bytes) + " bytes, expected " +
                   std::to_string(sizeof(curc::learned::Model));
        return CURC_ERR_ARG;
    }
    auto m = std::make_unique<curc::learned::Model>();
    std::memcpy(m.get(), model, sizeof(curc::learned::Model));
    ctx->mismatch_model = std::move(m);
    return CURC_OK;
}

extern "C" int curc_compress_files(curc_ctx* ctx, const char* f1, const char* f2, const char* archive_path,
                                   double block_ratio, int preserve_order, int flzma2_level, int flzma2_threads,
                                   const char* bsc_path, const char* tmpdir, uint64_t* reads_out,
                                   uint32_t* blocks_out) {
    if (!ctx || !f1 || !archive_path || !bsc_path || !tmpdir) return CURC_ERR_ARG;
    if (!(block_ratio > 0 && block_ratio <= 1)) {
        ctx->err = "block ratio is a float number in the range (0,1]";
        return CURC_ERR_ARG;
    }
    try {
        // a deferred context is not waited for here: the sink parses while
        // its CUDA set-up runs (DeviceSink)
        if (!ctx->ready.valid()) CURC_CHECK(cudaSetDevice(ctx->device));
        curc::host::CoderParams cp;
        cp.flzma2_level = flzma2_level;
        cp.flzma2_threads = flzma2_threads;
        cp.bsc_path = bsc_path;
        cp.tmpdir = tmpdir;
        const std::string s2 = f2 ? f2 : "";
        // CURC_VERBOSE=1 prints host-side stage times to stderr
        const bool verbose = std::getenv("CURC_VERBOSE") != nullptr;
        const auto t0 = std::chrono::steady_clock::now();
        curc::FileTimes times;
        curc::DeviceSink sink(ctx, preserve_order != 0, !s2.empty(), cp, verbose, times, ctx->mismatch_model.get());
        const auto res = curc::host::ingest_fastq(f1, s2, block_ratio, sink);
        const auto t1 = std::chrono::steady_clock::now();
        const int L = res.read_len;
        auto& bodies = sink.bodies;
        // the block (an input without reads never attached the sink)
        if (const int rc = curc::ctx_wait(ctx)) return rc;
        curc::Block& blk = *ctx->block;
        FILE* out = std::fopen(archive_path, "wb");
        if (!out) throw std::runtime_error(std::string("cannot write ") + archive_path);
        const std::string hdr = curc::host::archive_header(preserve_order != 0, !s2.empty(), L, res.blocks);
        std::fwrite(hdr.data(), 1, hdr.size(), out);
        for (auto& f : bodies) {
            const std::string b = f.get();
            std::fwrite(b.data(), 1, b.size(), out);
        }
        std::fclose(out);
        const auto t2 = std::chrono::steady_clock::now();
        auto ms = [](std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
            return float(std::chrono::duration<double, std::milli>(b - a).count());
        };
        if (verbose) std::fprintf(stderr, "curc: total %.3f s\n", ms(t0, t2) / 1000.0);
        // host-stage times of this call, readable with curc_block_stage_ms
        blk.stage_ms["files.total"] = ms(t0, t2);
        blk.stage_ms["files.until_last_block"] = ms(t0, t1);
        blk.stage_ms["files.coder_tail"] = ms(t1, t2);
        {
            std::lock_guard<std::mutex> g(times.mu);
            blk.stage_ms["files.ingest"] = float(times.ingest * 1000.0);
            blk.stage_ms["files.device"] = float(times.device * 1000.0);
            blk.stage_ms["files.snapshot"] = float(times.snapshot * 1000.0);
            blk.stage_ms["files.coders"] = float(times.coders * 1000.0);
            for (const auto& kv : times.coder) blk.stage_ms["coder." + kv.first] = float(kv.second * 1000.0);
            if (ctx->mismatch_model) {
                // learned mode: mismatch-stream kilobytes of each coding and
                // the blocks that kept the learned one
                blk.stage_ms["files.mismatch_plain_kb"] = float(double(times.mis_plain) / 1000.0);
                blk.stage_ms["files.mismatch_learned_kb"] = float(double(times.mis_learned) / 1000.0);
                blk.stage_ms["files.learned_blocks"] = float(times.learned_blocks);
            }
        }
        if (reads_out) *reads_out = res.reads;
        if (blocks_out) *blocks_out = uint32_t(res.blocks);
        return CURC_OK;
    } catch (const curc::CudaError& e) {
        ctx->err = e.what();
        return CURC_ERR_CUDA;
    } catch (const std::exception& e) {
        ctx->err = e.what();
        return CURC_ERR_IO;
    }
}
