// Block stream coding and the .curc archive layout.
//
// Layout (must match the reference byte for byte; read by decompress.cu:
// 760-814): archive header `u8 preserve_order, u8 paired_end, u16 read_len,
// u8 blocks` (preprocess.cpp:261-266), then each block body: `u32 reads`,
// 16-byte mismatch decoder table, [PO: u8 joined-length-fits-u32], u8
// ref-length-fits-u32, three u64 pseudogenome lengths, then u64-length-
// prefixed payloads in the order of compress.cu:2112-2146.
//
// The coders are the reference's vendored third-party libraries, linked
// unmodified: fast-lzma2 (pseudogenome, positions), the LZMA SDK with PPMd7
// and PgRC's VarLenDNACoder, the CLR range coder (mismatch offsets), and the
// `bsc` executable built from libbsc (strand stream, run as a subprocess
// exactly as util.cuh:527-535 does).  Independent streams, and the
// sub-streams of the position and pair-order coders, are coded concurrently:
// the LZMA / PPMd7 container of LzmaLib.cpp is restated here over the LZMA
// SDK's encoders (the library's own entry point also writes to a shared log
// stream, which concurrent callers would race on).
#include <sys/stat.h>
#include <unistd.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <future>
#include <mutex>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#ifndef ABS
#define ABS std::abs
#endif
#include <fast-lzma2/fast-lzma2.h>
#include <lzma/Alloc.h>
#include <lzma/LzmaEnc.h>
#include <lzma/Ppmd7.h>
#include <lzma/VarLenDNACoder/LzmaLib.h>
#include <range_coder/clr.cdr>
#include <range_coder/simple_model.h>

#include "../../../include/curc_b200.h"
#include "host.hpp"
#include "stable_order.hpp"

namespace curc {
namespace host {

namespace {

// PPMd7 coded bytes as LzmaLib.cpp:229-264 writes them at level 3
// (PGRC_CODER_LEVEL_MAX): 5 property bytes (model order, u32 memory size),
// then the range coder's output.  The memory size is 192 MiB shrunk to the
// smallest power of two 2^16..2^31 that is at least 16 times the input
// (LzmaLib.cpp:118-159).
struct ByteSink {
    IByteOut vt;
    std::string* out;
    static void put(const IByteOut* p, Byte b) {
        reinterpret_cast<const ByteSink*>(p)->out->push_back(char(b));
    }
};

std::string ppmd7_coded(const uint8_t* src, size_t n, int order) {
    uint32_t mem = 192u << 20;
    if (mem / 16 > n)
        for (unsigned i = 16; i <= 31; ++i) {
            const uint32_t m = 1u << i;
            if (n <= m / 16) {
                if (mem > m) mem = m;
                break;
            }
        }
    CPpmd7 ppmd;
    Ppmd7_Construct(&ppmd);
    if (!Ppmd7_Alloc(&ppmd, mem, &g_Alloc)) throw std::runtime_error("PPMd7: out of memory");
    Ppmd7_Init(&ppmd, unsigned(order));
    std::string out(5, '\0');
    out[0] = char(order);
    std::memcpy(&out[1], &mem, 4);
    out.reserve(5 + n / 2 + 64);
    ByteSink sink{{&ByteSink::put}, &out};
    CPpmd7z_RangeEnc rc;
    Ppmd7z_RangeEnc_Init(&rc);
    rc.Stream = &sink.vt;
    for (size_t i = 0; i < n; ++i) Ppmd7_EncodeSymbol(&ppmd, &rc, src[i]);
    Ppmd7z_RangeEnc_FlushData(&rc);
    Ppmd7_Free(&ppmd, &g_Alloc);
    return out;
}

// LZMA coded bytes as LzmaLib.cpp:88-117 and :162-181 write them at level 3:
// level 9, dictionary 1.5 GiB (reduced to the input by the encoder), lc 3,
// lp = pb = the data period code, 273 fast bytes, 2 threads; 5 property
// bytes, then the stream.
std::string lzma_coded(const uint8_t* src, size_t n, int period, size_t bound) {
    CLzmaEncProps props;
    LzmaEncProps_Init(&props);
    props.level = 9;
    props.dictSize = 3u << 29;
    props.lc = 3;
    props.lp = period;
    props.pb = period;
    props.fb = 273;
    props.numThreads = 2;
    props.reduceSize = n;
    std::string out(bound, '\0');
    SizeT props_size = LZMA_PROPS_SIZE, len = bound - LZMA_PROPS_SIZE;
    const SRes r = LzmaEncode(reinterpret_cast<Byte*>(&out[LZMA_PROPS_SIZE]), &len, src, n, &props,
                              reinterpret_cast<Byte*>(&out[0]), &props_size, 0, nullptr, &g_Alloc, &g_Alloc);
    if (r != SZ_OK) throw std::runtime_error("LZMA: encoding failed (code " + std::to_string(r) + ")");
    out.resize(LZMA_PROPS_SIZE + len);
    return out;
}

// The LzmaLib container (writeCompressed, LzmaLib.cpp:539-552) at level 3:
// u64 input length; unless it is zero, u64 coded length, u8 coder type and
// the coded bytes.  The library sizes its output buffer from the caller's
// ratio estimate and fails (exits) when the coded bytes do not fit; the
// same bound makes that an error here.
std::string container(const void* src, size_t n, uint8_t coder, int param, double est) {
    std::string o(8, '\0');
    const uint64_t n64 = n;
    std::memcpy(&o[0], &n64, 8);
    if (n == 0) return o;
    const size_t bound = size_t(double(LZMA_PROPS_SIZE) + double(n + n / 3) * est + 128);
    const uint8_t* p = static_cast<const uint8_t*>(src);
    std::string coded;
    if (coder == PPMD7_CODER) {
        coded = ppmd7_coded(p, n, param);
        if (coded.size() > bound) throw std::runtime_error("PPMd7: coded stream above the container's bound");
    } else if (coder == LZMA_CODER) {
        coded = lzma_coded(p, n, param, bound);
    } else {
        throw std::runtime_error("unsupported container coder");
    }
    const uint64_t c64 = coded.size();
    o.append(reinterpret_cast<const char*>(&c64), 8);
    o.push_back(char(coder));
    return o + coded;
}

// Containers coded on concurrent threads, returned in order.
std::string containers(std::initializer_list<std::function<std::string()>> parts) {
    std::vector<std::future<std::string>> f;
    for (const auto& p : parts) f.push_back(std::async(std::launch::async, p));
    std::string o;
    for (auto& x : f) o += x.get();
    return o;
}

// fast-lzma2 stream with the feeding pattern of the reference's file helper
// (8 KiB input reads, 4 KiB output buffer), so the bytes are identical.
std::string fl2(const void* data, size_t n, int level, int threads) {
    FL2_CStream* cs = FL2_createCStreamMt(unsigned(threads), 0);
    if (!cs) throw std::runtime_error("fast-lzma2: cannot create a compression context");
    size_t r = FL2_initCStream(cs, level);
    if (FL2_isError(r)) throw std::runtime_error(std::string("fast-lzma2: ") + FL2_getErrorName(r));
    const unsigned char* src = static_cast<const unsigned char*>(data);
    size_t consumed = 0;
    unsigned char in_buffer[8 * 1024];
    unsigned char out_buffer[4 * 1024];
    FL2_inBuffer in = {in_buffer, sizeof(in_buffer), sizeof(in_buffer)};
    FL2_outBuffer out = {out_buffer, sizeof(out_buffer), 0};
    std::string res;
    do {
        if (in.pos == in.size) {
            const size_t take = std::min(sizeof(in_buffer), n - consumed);
            std::memcpy(in_buffer, src + consumed, take);
            consumed += take;
            in.size = take;
            in.pos = 0;
        }
        r = FL2_compressStream(cs, &out, &in);
        if (FL2_isError(r)) throw std::runtime_error(std::string("fast-lzma2: ") + FL2_getErrorName(r));
        res.append(reinterpret_cast<const char*>(out_buffer), out.pos);
        out.pos = 0;
    } while (in.size == sizeof(in_buffer));
    do {
        r = FL2_endStream(cs, &out);
        if (FL2_isError(r)) throw std::runtime_error(std::string("fast-lzma2: ") + FL2_getErrorName(r));
        res.append(reinterpret_cast<const char*>(out_buffer), out.pos);
        out.pos = 0;
    } while (r);
    FL2_freeCStream(cs);
    return res;
}

std::string blob(const std::string& s) {
    std::string o(8, '\0');
    const uint64_t n = s.size();
    std::memcpy(&o[0], &n, 8);
    return o + s;
}

template <size_t MaxL>
std::string offsets_coded(const uint16_t* a, size_t count, size_t m) {
    // util.cuh:307-343
    std::vector<char> buf(count * sizeof(uint16_t) + 1024);
    RangeCoder rc{};
    rc.output(buf.data());
    rc.StartEncode();
    SIMPLE_MODEL<2> flag;
    SIMPLE_MODEL<MaxL / 2 + 1> first;
    SIMPLE_MODEL<MaxL> value;
    size_t i = 0;
    while (i < count) {
        flag.encodeSymbol(&rc, a[i++]);
        first.encodeSymbol(&rc, a[i++]);
        if (m > 1) {
            value.encodeSymbol(&rc, a[i++]);
            if (m > 2)
                for (size_t k = 1; k < m; ++k) value.encodeSymbol(&rc, a[i++]);
        }
    }
    rc.FinishEncode();
    return std::string(buf.data(), rc.size_out());
}

std::string offsets(int L, const uint16_t* a, size_t count, size_t m) {
    if (L <= 128) return offsets_coded<128>(a, count, m);
    if (L <= 256) return offsets_coded<256>(a, count, m);
    if (L <= 384) return offsets_coded<384>(a, count, m);
    return offsets_coded<512>(a, count, m);
}

std::string read_file(const std::string& p) {
    FILE* f = std::fopen(p.c_str(), "rb");
    if (!f) throw std::runtime_error("cannot open " + p);
    std::string s;
    char buf[1 << 16];
    size_t k;
    while ((k = std::fread(buf, 1, sizeof(buf), f)) > 0) s.append(buf, k);
    std::fclose(f);
    return s;
}

void write_file(const std::string& p, const void* d, size_t n) {
    FILE* f = std::fopen(p.c_str(), "wb");
    if (!f) throw std::runtime_error("cannot write " + p);
    if (n && std::fwrite(d, 1, n, f) != n) throw std::runtime_error("short write " + p);
    std::fclose(f);
}

// libbsc through its executable (util.cuh:527-535 runs it so for the strand
// stream): `bsc e in out -pm0 -e2`.
std::string bsc_strand(const std::string& bsc, const std::string& dir, const void* d, size_t n) {
    static std::atomic<uint64_t> seq{0};
    const std::string tag = std::to_string(getpid()) + "_" + std::to_string(seq.fetch_add(1));
    const std::string in = dir + "/strand_" + tag + ".txt", out = dir + "/strand_" + tag + ".bsc";
    write_file(in, d, n);
    const std::string cmd = "'" + bsc + "' e '" + in + "' '" + out + "' -pm0 -e2 > /dev/null";
    if (std::system(cmd.c_str()) != 0) throw std::runtime_error("bsc failed: " + cmd);
    std::string s = read_file(out);
    unlink(in.c_str());
    unlink(out.c_str());
    return s;
}

template <class T>
std::string pe_id_to_pos(const uint64_t* id_to_pos, size_t n, int level, int thr, const CoderParams& cp) {
    // util.cuh:345-442
    using clk = std::chrono::steady_clock;
    static const bool verbose = std::getenv("CURC_VERBOSE") != nullptr;
    auto mark = [&](const char* what, clk::time_point a) {
        const double sec = std::chrono::duration<double>(clk::now() - a).count();
        if (verbose) std::fprintf(stderr, "curc:   coder %-16s %.3f s\n", what, sec);
        if (cp.on_time) cp.on_time(what, sec);
    };
    std::vector<T> base, notbase;
    std::vector<uint8_t> off_flag, off_first, d_flag, d_first;
    std::vector<uint16_t> off_val;
    std::vector<int16_t> d_val;
    const uint32_t pairs = uint32_t(n / 2);
    base.reserve(pairs);
    for (uint32_t i = 0; i < n; i += 2) base.push_back(T(id_to_pos[i]));
    // the first mates' positions are coded as they are: their fast-lzma2
    // stream runs while the pairs are ordered and split
    auto fb = std::async(std::launch::async, [&] {
        const auto a = clk::now();
        std::string r = fl2(base.data(), base.size() * sizeof(T), level, thr);
        mark("id_pos.fl2_base", a);
        return r;
    });
    auto t = clk::now();
    // pairs by their first mate's position, ties in pair order (the
    // reference's stable sort, on host threads)
    const std::vector<uint32_t> rank = stable_order(base.data(), base.size(), thr);
    mark("id_pos.order", t);
    t = clk::now();
    // per pair, in that order: which mate comes first and their distance,
    // read on host threads (the second mates' positions are read at random);
    // the pairs within 16 bits go to their streams by a prefix count, the
    // others, which carry the delta coder's state, in one pass
    const size_t nt = chunk_count(pairs, thr);
    std::vector<uint8_t> bef(pairs);
    std::vector<T> relv(pairs);
    off_flag.resize(pairs);
    std::vector<size_t> n16(nt + 1, 0);
    each_chunk(pairs, nt, [&](size_t lo, size_t hi, size_t c) {
        size_t k = 0;
        for (size_t q = lo; q < hi; ++q) {
            const uint32_t i = rank[q] * 2;
            const bool before = id_to_pos[i] < id_to_pos[i + 1];
            const T rel = before ? T(id_to_pos[i + 1] - id_to_pos[i]) : T(id_to_pos[i] - id_to_pos[i + 1]);
            bef[q] = before;
            relv[q] = rel;
            off_flag[q] = rel <= 0xFFFF;
            k += off_flag[q];
        }
        n16[c + 1] = k;
    });
    for (size_t c = 0; c < nt; ++c) n16[c + 1] += n16[c];
    off_first.resize(n16[nt]);
    off_val.resize(n16[nt]);
    each_chunk(pairs, nt, [&](size_t lo, size_t hi, size_t c) {
        size_t p = n16[c];
        for (size_t q = lo; q < hi; ++q)
            if (off_flag[q]) {
                off_first[p] = bef[q];
                off_val[p] = uint16_t(relv[q]);
                ++p;
            }
    });
    int64_t ref_prev = 0, prev = 0;
    bool match = false;
    for (uint32_t q = 0; q < pairs; ++q) {
        if (off_flag[q]) continue;
        const uint32_t i = rank[q] * 2;
        const bool before = bef[q] != 0;
        const T rel = relv[q];
        const int64_t delta = int64_t(rel) - ref_prev;
        const bool d16 = delta <= INT16_MAX && delta >= INT16_MIN;
        d_flag.push_back(d16);
        if (d16) {
            match = true;
            d_first.push_back(before);
            d_val.push_back(int16_t(delta));
            ref_prev = int64_t(rel);
        } else {
            if (!match || ref_prev != prev) ref_prev = int64_t(rel);
            notbase.push_back(T(id_to_pos[i + 1]));
            match = false;
        }
        prev = int64_t(rel);
    }
    mark("id_pos.split", t);
    auto fn = std::async(std::launch::async, [&] { return fl2(notbase.data(), notbase.size() * sizeof(T), level, thr); });
    const double bm = COMPRESSION_ESTIMATION_UINT8_BITMAP;
    t = clk::now();
    std::string mid = containers({
        [&] { return container(off_flag.data(), off_flag.size(), PPMD7_CODER, 3, bm); },
        [&] { return container(off_first.data(), off_first.size(), PPMD7_CODER, 3, bm); },
        [&] { return container(off_val.data(), off_val.size() * 2, PPMD7_CODER, 3, 1); },
        [&] { return container(d_flag.data(), d_flag.size(), PPMD7_CODER, 3, bm); },
        [&] { return container(d_first.data(), d_first.size(), PPMD7_CODER, 3, bm); },
        [&] { return container(d_val.data(), d_val.size() * 2, PPMD7_CODER, 3, 1); },
    });
    mark("id_pos.ppmd", t);
    std::string o = blob(fb.get());
    o += mid;
    o += blob(fn.get());
    return o;
}

std::string pe_order(const uint32_t* order, size_t n, int level, int thr) {
    // util.cuh:444-525
    std::vector<uint8_t> off_pair, non_off_pair, off8_flag, off8_val, d8_flag;
    std::vector<int8_t> d8_val;
    std::vector<uint32_t> offs;
    std::vector<uint8_t> visit(n, 0);
    std::vector<uint32_t> index(n);
    for (uint32_t i = 0; i < n; ++i) index[order[i]] = i;
    int64_t ref_prev = 0, prev = 0;
    bool match = false;
    for (uint32_t oi = 0; oi < n; ++oi) {
        if (visit[oi]) continue;
        const uint32_t o = order[oi];
        const uint32_t po = o % 2 ? o - 1 : o + 1;
        const uint32_t pi = index[po];
        visit[pi] = 1;
        const int64_t d = int64_t(pi) - int64_t(oi);
        off8_flag.push_back(d <= 255);
        if (d <= 255) {
            off8_val.push_back(uint8_t(d));
            off_pair.push_back(o % 2);
            continue;
        }
        non_off_pair.push_back(o % 2);
        const int64_t delta = d - ref_prev;
        const bool d8 = delta >= INT8_MIN && delta <= INT8_MAX;
        d8_flag.push_back(d8);
        if (d8) {
            match = true;
            d8_val.push_back(int8_t(delta));
            ref_prev = d;
        } else {
            if (!match || ref_prev != prev) ref_prev = d;
            offs.push_back(uint32_t(d));
            match = false;
        }
        prev = d;
    }
    auto fd = std::async(std::launch::async, [&] { return fl2(d8_val.data(), d8_val.size(), level, thr); });
    auto fo = std::async(std::launch::async, [&] { return fl2(offs.data(), offs.size() * 4, level, thr); });
    const double bm = COMPRESSION_ESTIMATION_UINT8_BITMAP;
    std::string out = containers({
        [&] { return container(off8_flag.data(), off8_flag.size(), PPMD7_CODER, 3, bm); },
        [&] { return container(off8_val.data(), off8_val.size(), PPMD7_CODER, 2, 1); },
        [&] { return container(d8_flag.data(), d8_flag.size(), PPMD7_CODER, 3, bm); },
        [&] { return container(off_pair.data(), off_pair.size(), PPMD7_CODER, 2, bm); },
        [&] { return container(non_off_pair.data(), non_off_pair.size(), PPMD7_CODER, 2, bm); },
    });
    out += blob(fd.get());
    out += blob(fo.get());
    return out;
}

}  // namespace

// CURC_VERBOSE=1: time of each coder on stderr.
template <class F>
std::string timed(const CoderParams& cp, const char* what, F&& f) {
    static const bool verbose = std::getenv("CURC_VERBOSE") != nullptr;
    const auto t0 = std::chrono::steady_clock::now();
    std::string r = f();
    const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (verbose) std::fprintf(stderr, "curc:   coder %-16s %.3f s, %zu bytes\n", what, s, r.size());
    if (cp.on_time) cp.on_time(what, s);
    return r;
}

std::string encode_block(const BlockView& v, const CoderParams& cp) {
    const int L = v.read_len;
    const auto& S = [&](const char* name) -> const Buf& { return v.get(name); };
    std::string hdr;
    auto put = [&](const void* p, size_t n) { hdr.append(static_cast<const char*>(p), n); };
    put(&v.reads_count, 4);
    put(S("decoder_table").ptr, 16);
    const uint64_t* sizes = reinterpret_cast<const uint64_t*>(S("sizes").ptr);  // pre- and post-compaction
    const uint64_t joined = sizes[0] + sizes[1] + sizes[2];
    const uint8_t join_std = joined <= 0xFFFFFFFFull, ref_std = sizes[0] <= 0xFFFFFFFFull;
    if (v.preserve_order) put(&join_std, 1);
    put(&ref_std, 1);
    put(sizes + 3, 24);

    const int lvl = cp.flzma2_level, thr = cp.flzma2_threads;
    // concurrent coders
    std::future<std::string> f_idpos, f_strand, f_ref, f_peorder;
    if (v.preserve_order) {
        f_idpos = std::async(std::launch::async, [&] { return timed(cp, "id_pos", [&] {
            const Buf& b = S("id_to_pos");
            const uint64_t* p = reinterpret_cast<const uint64_t*>(b.ptr);
            const size_t n = b.size / 8;
            if (!v.paired_end) {
                if (join_std) {
                    std::vector<uint32_t> v32(p, p + n);
                    return fl2(v32.data(), v32.size() * 4, lvl, thr);
                }
                return fl2(p, n * 8, lvl, thr);
            }
            return join_std ? pe_id_to_pos<uint32_t>(p, n, lvl, thr, cp) : pe_id_to_pos<uint64_t>(p, n, lvl, thr, cp);
        }); });
    }
    f_strand = std::async(std::launch::async, [&] { return timed(cp, "strand", [&] {
        const Buf& b = S("strand");
        return bsc_strand(cp.bsc_path, cp.tmpdir, b.ptr, b.size);
    }); });
    f_ref = std::async(std::launch::async, [&] { return timed(cp, "ref", [&] {
        std::string joined_ref;
        joined_ref.reserve(S("ref").size + S("unmap_ref").size + S("unmap_n_ref").size);
        for (const char* nm : {"ref", "unmap_ref", "unmap_n_ref"})
            joined_ref.append(reinterpret_cast<const char*>(S(nm).ptr), S(nm).size);
        // compress.cu:2099-2102: the VarLenDNA coder (called directly; it
        // keeps no shared state), then fast-lzma2
        size_t clen = 0;
        unsigned char* enc = nullptr;
        const int rc = PgSAHelpers::VarLenDNACoder::Compress(
            enc, clen, reinterpret_cast<const unsigned char*>(joined_ref.data()), joined_ref.size(),
            PgSAHelpers::VarLenDNACoder::getCoderParam(PgSAHelpers::VarLenDNACoder::STATIC_CODES_CODER_PARAM,
                                                       PgSAHelpers::VarLenDNACoder::AG_EXTENDED_CODES_ID));
        if (rc != SZ_OK) {
            delete[] enc;
            throw std::runtime_error("VarLenDNA coder failed");
        }
        std::string r = fl2(enc, clen, lvl, thr);
        delete[] enc;
        return r;
    }); });
    if (!v.preserve_order && v.paired_end) {
        f_peorder = std::async(std::launch::async, [&] { return timed(cp, "pe_order", [&] {
            const Buf& b = S("pe_order");
            return pe_order(reinterpret_cast<const uint32_t*>(b.ptr), b.size / 4, lvl, thr);
        }); });
    }
    // mismatch offsets (CLR range coder) in parallel per class
    const int max_mm = L / 5;
    std::vector<std::future<std::string>> f_off;
    for (int m = 1; m <= max_mm; ++m) {
        f_off.push_back(std::async(std::launch::async, [&, m] { return timed(cp, "mis_off", [&] {
            const Buf& b = S(("mis_off_" + std::to_string(m)).c_str());
            return offsets(L, reinterpret_cast<const uint16_t*>(b.ptr), b.size / 2, size_t(m));
        }); }));
    }
    // the PPMd7 / LZMA container streams, each on its own thread
    auto plain = [&](const char* what, const char* nm, uint8_t coder, int param, double est) {
        return std::async(std::launch::async, [&, what, nm, coder, param, est] {
            return timed(cp, what, [&] {
                const Buf& b = S(nm);
                return container(b.ptr, b.size, coder, param, est);
            });
        });
    };
    std::future<std::string> read_off, unmap_n_off, unmap_off;
    if (!v.preserve_order) {
        read_off = plain("read_off", "read_off", PPMD7_CODER, 3, 1);
        unmap_n_off = plain("read_off", "unmap_n_read_off", PPMD7_CODER, 3, 1);
        unmap_off = plain("read_off", "unmap_read_off", PPMD7_CODER, 3, 1);
    }
    const double est = simpleUintCompressionEstimate(S("ref").size, ref_std ? 0xFFFFFFFFull : ~0ull);
    const int period = ref_std ? 2 : 3;
    std::vector<std::future<std::string>> maps;
    for (auto pr : {std::make_pair("ref_off", "ref_len_map"), std::make_pair("unmap_ref_off", "unmap_ref_len"),
                    std::make_pair("unmap_n_ref_off", "unmap_n_ref_len")}) {
        maps.push_back(plain("maps", pr.first, LZMA_CODER, period, est));
        maps.push_back(plain("maps", pr.second, LZMA_CODER, 0, 1));
    }
    auto mis_cnt = plain("mis_cnt", "mis_cnt", PPMD7_CODER, 2, 1);
    auto mis_base = plain("mis_base", "mis_base", PPMD7_CODER, 2, COMPRESSION_ESTIMATION_MIS_SYM);

    std::string out = hdr;
    if (v.preserve_order) out += blob(f_idpos.get());
    out += blob(f_strand.get());
    out += blob(f_ref.get());
    if (!v.preserve_order) {
        out += blob(read_off.get());
        out += blob(unmap_n_off.get());
        out += blob(unmap_off.get());
        if (v.paired_end) out += blob(f_peorder.get());
    }
    for (auto& m : maps) out += blob(m.get());
    out += blob(mis_cnt.get());
    const uint8_t mm = uint8_t(max_mm);
    std::string tail = blob(mis_base.get());
    tail.append(reinterpret_cast<const char*>(&mm), 1);
    for (auto& f : f_off) tail += blob(f.get());
    if (!v.learned_stream.empty()) {
        // learned mode: the mismatch-base container holds, under the coder
        // byte LEARNED_CODER, the model and the learned stream of bases and
        // offsets together; the offset streams are then empty.  Kept only
        // where it is smaller than the plain coding of the same streams.
        std::string c(17, '\0');
        const uint64_t src = S("mis_base").size;
        const uint64_t clen = 4 + v.learned_model.size() + v.learned_stream.size();
        std::memcpy(&c[0], &src, 8);
        std::memcpy(&c[8], &clen, 8);
        c[16] = char(LEARNED_CODER);
        const uint32_t msize = uint32_t(v.learned_model.size());
        c.append(reinterpret_cast<const char*>(&msize), 4);
        c += v.learned_model;
        c += v.learned_stream;
        std::string lt = blob(c);
        lt.append(reinterpret_cast<const char*>(&mm), 1);
        lt.append(size_t(max_mm) * 8, '\0');
        if (cp.on_learned) cp.on_learned(tail.size(), lt.size());
        if (lt.size() < tail.size()) tail.swap(lt);
    }
    out += tail;
    return out;
}

void plain_mismatch_bytes(const BlockView& v, uint64_t out[3]) {
    const int L = v.read_len;
    out[0] = container(v.get("mis_cnt").ptr, v.get("mis_cnt").size, PPMD7_CODER, 2, 1).size();
    out[1] = container(v.get("mis_base").ptr, v.get("mis_base").size, PPMD7_CODER, 2,
                       COMPRESSION_ESTIMATION_MIS_SYM).size();
    uint64_t o = 0;
    for (int m = 1; m <= L / 5; ++m) {
        const Buf& b = v.get(("mis_off_" + std::to_string(m)).c_str());
        o += offsets(L, reinterpret_cast<const uint16_t*>(b.ptr), b.size / 2, size_t(m)).size();
    }
    out[2] = o;
}

void general_mismatch_bytes(const BlockView& v, const CoderParams& cp, uint64_t out[2]) {
    // the three raw mismatch streams: counts, recoded bases, and the offset
    // values of every count class one after another
    const int L = v.read_len;
    std::string offs;
    for (int m = 1; m <= L / 5; ++m) {
        const Buf& b = v.get(("mis_off_" + std::to_string(m)).c_str());
        offs.append(reinterpret_cast<const char*>(b.ptr), b.size);
    }
    const Buf& c = v.get("mis_cnt");
    const Buf& b = v.get("mis_base");
    const std::pair<const void*, size_t> streams[3] = {{c.ptr, c.size}, {b.ptr, b.size}, {offs.data(), offs.size()}};
    out[0] = out[1] = 0;
    for (const auto& st : streams) {
        if (!st.second) continue;
        out[0] += fl2(st.first, st.second, cp.flzma2_level, cp.flzma2_threads).size();
        out[1] += bsc_strand(cp.bsc_path, cp.tmpdir, st.first, st.second).size();
    }
}

std::string archive_header(bool po, bool pe, int read_len, int blocks) {
    std::string h(5, '\0');
    h[0] = char(po);
    h[1] = char(pe);
    h[2] = char(read_len & 0xFF);
    h[3] = char(read_len >> 8);
    h[4] = char(blocks);
    return h;
}

}  // namespace host
}  // namespace curc

namespace curc {
std::string& ctxless_error();
}

extern "C" {

int curc_encode_block(uint32_t reads_count, uint16_t read_len, int preserve_order, int paired_end,
                      const char* const* names, const void* const* ptrs, const uint64_t* sizes, uint32_t count,
                      int flzma2_level, int flzma2_threads, const char* bsc_path, const char* tmpdir, char** out,
                      uint64_t* out_bytes) {
    if (!out || !out_bytes || !bsc_path || !tmpdir || (count && (!names || !ptrs || !sizes)) || read_len < 1 ||
        read_len > 511) {
        curc::ctxless_error() = "curc_encode_block: bad argument";
        return CURC_ERR_ARG;
    }
    *out = nullptr;
    *out_bytes = 0;
    try {
        curc::host::BlockView v;
        v.reads_count = reads_count;
        v.read_len = read_len;
        v.preserve_order = preserve_order != 0;
        v.paired_end = paired_end != 0;
        for (uint32_t i = 0; i < count; ++i) {
            if (!names[i] || (sizes[i] && !ptrs[i])) throw std::invalid_argument("curc_encode_block: null stream");
            v.streams[names[i]] = curc::host::Buf{static_cast<const uint8_t*>(ptrs[i]), size_t(sizes[i])};
        }
        curc::host::CoderParams cp;
        cp.flzma2_level = flzma2_level;
        cp.flzma2_threads = flzma2_threads;
        cp.bsc_path = bsc_path;
        cp.tmpdir = tmpdir;
        const std::string body = curc::host::encode_block(v, cp);
        char* b = static_cast<char*>(std::malloc(body.size() ? body.size() : 1));
        if (!b) throw std::bad_alloc();
        std::memcpy(b, body.data(), body.size());
        *out = b;
        *out_bytes = body.size();
        return CURC_OK;
    } catch (const std::invalid_argument& e) {
        curc::ctxless_error() = e.what();
        return CURC_ERR_ARG;
    } catch (const std::exception& e) {
        curc::ctxless_error() = e.what();
        return CURC_ERR_STATE;
    }
}

void curc_buffer_free(char* p) { std::free(p); }

int curc_archive_header(int preserve_order, int paired_end, uint16_t read_len, uint32_t blocks, char* out5) {
    if (!out5 || blocks > 254 || read_len < 1 || read_len > 511) {
        curc::ctxless_error() = "curc_archive_header: bad argument";
        return CURC_ERR_ARG;
    }
    const std::string h = curc::host::archive_header(preserve_order != 0, paired_end != 0, read_len, int(blocks));
    std::memcpy(out5, h.data(), 5);
    return CURC_OK;
}

}  // extern "C"
