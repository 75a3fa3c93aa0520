// Whole-file compression through the device path: FASTQ ingest, one block
// run per block, stream coding on host threads overlapped with the next
// block's ingest and device work, archive in the reference layout
// (the reference's process() + block_compress(), preprocess.cpp:66-283).
#include <unistd.h>

#include <cstdio>
#include <future>
#include <memory>
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
        std::vector<std::future<std::string>> bodies;
        int L = 0;
        auto res = curc::host::ingest_fastq(f1, s2, block_ratio, [&](std::vector<char>&& seqs, uint64_t n, int len) {
            L = len;
            blk.arena.reset();
            const size_t bytes = size_t(n) * len;
            uint8_t* d = blk.arena.alloc<uint8_t>(bytes + 16);
            if (bytes) CURC_CHECK(cudaMemcpyAsync(d, seqs.data(), bytes, cudaMemcpyHostToDevice, blk.stream));
            blk.run(d, n, len, preserve_order != 0, !s2.empty());
            auto snap = curc::snapshot(blk);
            bodies.push_back(std::async(std::launch::async, [snap, cp] { return curc::host::encode_block(snap->view, cp); }));
        });
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
