// Autotuner for the launch and table choices that change no result (no
// counterpart in the reference, whose launch shapes are Thrust defaults).
//
// Knobs (struct Tuning): the overlap index's bucket table size as a multiple
// of the prefix count, bits of the prefix presence bitmap per prefix, overlap
// passes between host reads of the link count, threads per block of the
// mapping kernel, and the form of the full-match pass loop (a launch per
// kernel, one graph, or one persistent kernel).  None of them changes which prefixes a suffix meets, the
// order candidates are visited in, or any stream: the tests compare every
// stage result and stream under each setting.  The k-mer length and the
// other derived parameters (preprocess.cpp:295-313) are part of the format
// and are never tuned.
//
// Search: coordinate descent on the caller's block, one knob at a time in
// the order above, each candidate timed by the device time of the stage it
// affects (best of two runs).  Choices are cached per (read length, read
// count rounded down to a power of two) in a small text file, one line per
// bucket: "L log2n table_factor bitmap_bits check_every map_threads
// fm_loop" (lines without the last field take its default).
#include <cmath>
#include <cstdio>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/curc_b200.h"
#include "block.cuh"

namespace curc {
namespace {

using Key = TuneKey;

std::map<Key, Tuning> load_cache(const std::string& path) {
    std::map<Key, Tuning> m;
    std::ifstream in(path);
    std::string line;
    while (std::getline(in, line)) {
        std::istringstream ls(line);
        Key k;
        Tuning t;
        if (!(ls >> k.L >> k.log2n >> t.table_factor >> t.bitmap_bits >> t.check_every >> t.map_threads)) continue;
        int g;
        if (ls >> g) t.fm_loop = g;
        m[k] = t;
    }
    return m;
}

void save_cache(const std::string& path, const std::map<Key, Tuning>& m) {
    const std::string tmp = path + ".tmp";
    {
        std::ofstream out(tmp, std::ios::trunc);
        for (const auto& kv : m)
            out << kv.first.L << ' ' << kv.first.log2n << ' ' << kv.second.table_factor << ' ' << kv.second.bitmap_bits
                << ' ' << kv.second.check_every << ' ' << kv.second.map_threads << ' ' << kv.second.fm_loop
                << '\n';
        if (!out) throw std::runtime_error("autotune: cannot write " + tmp);
    }
    if (std::rename(tmp.c_str(), path.c_str()) != 0) throw std::runtime_error("autotune: cannot replace " + path);
}

bool valid(const Tuning& t) {
    auto in = [](int v, std::initializer_list<int> ok) {
        for (int x : ok)
            if (v == x) return true;
        return false;
    };
    return in(t.table_factor, {1, 2, 4, 8}) && in(t.bitmap_bits, {8, 16, 32}) && in(t.check_every, {2, 4, 8, 16}) &&
           in(t.map_threads, {64, 128, 256}) && in(t.fm_loop, {0, 1, 2});
}

}  // namespace
}  // namespace curc

using curc::Tuning;

extern "C" {

int curc_ctx_set_tuning(curc_ctx* ctx, const int32_t* knobs) {
    if (!ctx || !knobs) return CURC_ERR_ARG;
    if (ctx)
        if (const int rc = curc::ctx_wait(ctx)) return rc;
    Tuning t{knobs[0], knobs[1], knobs[2], knobs[3], knobs[4]};
    if (!curc::valid(t)) {
        ctx->err = "tuning: a knob outside its candidate values";
        return CURC_ERR_ARG;
    }
    ctx->block->tune = t;
    return CURC_OK;
}

int curc_ctx_get_tuning(curc_ctx* ctx, int32_t* knobs) {
    if (!ctx || !knobs) return CURC_ERR_ARG;
    if (ctx)
        if (const int rc = curc::ctx_wait(ctx)) return rc;
    const Tuning& t = ctx->block->tune;
    knobs[0] = t.table_factor;
    knobs[1] = t.bitmap_bits;
    knobs[2] = t.check_every;
    knobs[3] = t.map_threads;
    knobs[4] = t.fm_loop;
    return CURC_OK;
}

int curc_ctx_use_tuning_cache(curc_ctx* ctx, const char* cache_path) {
    if (!ctx) return CURC_ERR_ARG;
    if (ctx)
        if (const int rc = curc::ctx_wait(ctx)) return rc;
    try {
        if (!cache_path || !*cache_path) {
            ctx->block->tune_cache.reset();
            return CURC_OK;
        }
        auto m = std::make_shared<std::map<curc::Key, Tuning>>();
        for (const auto& kv : curc::load_cache(cache_path))
            if (curc::valid(kv.second)) (*m)[kv.first] = kv.second;
        ctx->block->tune_cache = m;
        return CURC_OK;
    } catch (const std::exception& e) {
        ctx->err = e.what();
        return CURC_ERR_IO;
    }
}

int curc_autotune(curc_ctx* ctx, const char* seqs_dev, uint64_t n, uint16_t read_len, int preserve_order,
                  int paired_end, const char* cache_path, int* from_cache) {
    if (!ctx || !seqs_dev || !n) return CURC_ERR_ARG;
    if (ctx)
        if (const int rc = curc::ctx_wait(ctx)) return rc;
    try {
        CURC_CHECK(cudaSetDevice(ctx->device));
        curc::Block& blk = *ctx->block;
        const curc::Key key = curc::tune_key(int(read_len), n);
        std::map<curc::Key, Tuning> cache;
        if (cache_path && *cache_path) cache = curc::load_cache(cache_path);
        auto hit = cache.find(key);
        if (hit != cache.end() && curc::valid(hit->second)) {
            blk.tune = hit->second;
            if (from_cache) *from_cache = 1;
            return CURC_OK;
        }
        struct Restore {  // on every exit: intermediates as they were, tuning as chosen
            curc::Block& b;
            bool keep;
            Tuning t;
            ~Restore() {
                b.keep_intermediates = keep;
                b.tune = t;
            }
        } restore{blk, blk.keep_intermediates, blk.tune};
        blk.keep_intermediates = false;
        auto stage_time = [&](const Tuning& t, const char* stage) {
            blk.tune = t;
            float best = 1e30f;
            for (int r = 0; r < 2; ++r) {
                blk.arena.reset();  // the input is the caller's memory, not the arena's
                blk.run(reinterpret_cast<const uint8_t*>(seqs_dev), n, read_len, preserve_order != 0,
                        paired_end != 0);
                best = std::min(best, blk.stage_ms.at(stage));
            }
            return best;
        };
        Tuning best;
        struct Knob {
            int Tuning::*field;
            std::vector<int> values;
            const char* stage;
        };
        const Knob knobs[] = {{&Tuning::table_factor, {1, 2, 4, 8}, "overlap"},
                              {&Tuning::bitmap_bits, {8, 16, 32}, "overlap"},
                              {&Tuning::check_every, {4, 8, 16}, "overlap"},
                              {&Tuning::map_threads, {64, 128, 256}, "mapping"},
                              {&Tuning::fm_loop, {0, 1, 2}, "full_match"}};
        for (const Knob& k : knobs) {
            float tbest = 1e30f;
            int vbest = best.*(k.field);
            for (int v : k.values) {
                Tuning t = best;
                t.*(k.field) = v;
                const float ms = stage_time(t, k.stage);
                if (ms < tbest) {
                    tbest = ms;
                    vbest = v;
                }
            }
            best.*(k.field) = vbest;
        }
        restore.t = best;
        if (cache_path && *cache_path) {
            cache[key] = best;
            curc::save_cache(cache_path, cache);
        }
        if (from_cache) *from_cache = 0;
        return CURC_OK;
    } catch (const curc::CudaError& e) {
        ctx->err = e.what();
        return CURC_ERR_CUDA;
    } catch (const std::exception& e) {
        ctx->err = e.what();
        return CURC_ERR_STATE;
    }
}

}  // extern "C"
