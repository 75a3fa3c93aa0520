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

// Owned copy of a block's streams for the coder threads.
struct Snapshot {
    host::BlockView view;
    std::vector<std::vector<uint8_t>> store;
};

std::shared_ptr<Snapshot> snapshot(const Block& b) {
    auto s = std::make_shared<Snapshot>();
    s->view.reads_count = b.n;
    s->view.read_len = b.p.L;
    s->view.preserve_order = b.p.preserve_order;
    s->view.paired_end = b.p.paired_end;
    s->store.reserve(b.host.size());
    for (const auto& kv : b.host) {
        s->store.emplace_back(kv.second.ptr, kv.second.ptr + kv.second.size);
        s->view.streams[kv.first] = host::Buf{s->store.back().data(), s->store.back().size()};
    }
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

class DeviceSink : public host::IngestSink {
public:
    DeviceSink(Block& blk, bool po, bool pe, const host::CoderParams& cp, bool verbose, FileTimes& times,
               const learned::Model* model)
        : blk_(blk), po_(po), pe_(pe), cp_(cp), verbose_(verbose), times_(times), model_(model) {
        cp_.on_time = [t = &times_](const char* what, double s) { t->add_coder(what, s); };
        cp_.on_learned = [t = &times_](uint64_t plain, uint64_t learned) {
            std::lock_guard<std::mutex> g(t->mu);
            t->mis_plain += plain;
            t->mis_learned += learned;
            t->learned_blocks += learned < plain;
        };
        for (auto& e : ev_) CURC_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    ~DeviceSink() override {
        for (auto& e : ev_) cudaEventSynchronize(e);
        for (auto& e : ev_) cudaEventDestroy(e);
        for (auto& b : stage_)
            if (b.ptr) cudaFreeHost(b.ptr);
    }
    void begin_block(size_t max_bytes, int L) override {
        t_begin_ = clk::now();
        L_ = L;
        blk_.arena.reset();
        dev_ = blk_.arena.alloc<uint8_t>(max_bytes + 16);
        cap_ = max_bytes;
        off_ = 0;
        reads_ = 0;
    }
    char* window_buffer(size_t bytes) override {
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
        if (off_ + bytes > cap_) throw std::runtime_error("ingest: block larger than its bound");
        if (bytes)
            CURC_CHECK(cudaMemcpyAsync(dev_ + off_, stage_[cur_].ptr, bytes, cudaMemcpyHostToDevice, blk_.stream));
        CURC_CHECK(cudaEventRecord(ev_[cur_], blk_.stream));
        off_ += bytes;
        reads_ += reads;
    }
    void end_block() override {
        const auto ta = clk::now();
        blk_.run(dev_, reads_, L_, po_, pe_);
        const auto tb = clk::now();
        auto snap = snapshot(blk_);
        if (model_) {
            // learned mode: the block's learned mismatch stream, from the
            // block's device state before the next block reuses it; the
            // writer keeps it when it is smaller than the plain coding
            const auto l0 = clk::now();
            snap->view.learned_stream = learned::encode_stream(*model_, blk_);
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
    Block& blk_;
    bool po_, pe_;
    host::CoderParams cp_;
    bool verbose_;
    FileTimes& times_;
    const learned::Model* model_;
    Stage stage_[2];
    cudaEvent_t ev_[2];
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
        CURC_CHECK(cudaSetDevice(ctx->device));
        curc::Block& blk = *ctx->block;
        const bool keep_inter = blk.keep_intermediates;
        blk.keep_intermediates = false;
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
        curc::DeviceSink sink(blk, preserve_order != 0, !s2.empty(), cp, verbose, times, ctx->mismatch_model.get());
        const auto res = curc::host::ingest_fastq(f1, s2, block_ratio, sink);
        const auto t1 = std::chrono::steady_clock::now();
        const int L = res.read_len;
        auto& bodies = sink.bodies;
        blk.keep_intermediates = keep_inter;
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
