// Product decoder of `.curc` archives (`curc -d`): archive -> reads.
//
// Reference: decompress() and decompress_block() (decompress.cu:760-1060),
// with the stream readers of decompress.cu:59-416 and the read
// reconstruction of preserve_order_process (decompress.cu:462-566).  The
// archive layout is the one encode_block writes (compress.cu:1364-2146):
// the same vendored coders decode it (fast-lzma2, the LZMA SDK containers
// with PPMd7/LZMA, PgRC's VarLenDNACoder, the CLR range coder, bsc).
//
// Differences in shape, none in output: the block's streams are decoded in
// memory from the archive bytes (the reference writes each stream to a
// scratch file and reads it back; only bsc, an executable, still goes
// through files), and the reads are rebuilt by OpenMP over bounded output
// chunks written in the reference decoder's order.  The LZMA and PPMd
// payloads go straight to the LZMA SDK's decoders and the var-len DNA
// payload to a bounds-checked restatement, so a corrupt archive gives an
// error instead of ending the process (the vendored wrappers exit()).
#include <omp.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <future>
#include <numeric>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include <fast-lzma2/fast-lzma2.h>
#include <lzma/Alloc.h>
#include <lzma/LzmaDec.h>
#include <lzma/Ppmd7.h>
#include <lzma/VarLenDNACoder/LzmaLib.h>

#include "../../../include/curc_b200.h"
#include "host.hpp"
#include "stable_order.hpp"
#include "../learned_model.hpp"

namespace curc {
namespace host {

namespace {

// Bounds-checked little-endian reader over the archive bytes.
class Reader {
public:
    Reader(const std::string& s) : p_(reinterpret_cast<const uint8_t*>(s.data())), n_(s.size()) {}
    template <class T>
    T get() {
        need(sizeof(T));
        T v;
        std::memcpy(&v, p_ + off_, sizeof(T));
        off_ += sizeof(T);
        return v;
    }
    std::string bytes(size_t k) {
        need(k);
        std::string s(reinterpret_cast<const char*>(p_ + off_), k);
        off_ += k;
        return s;
    }
    // a size-prefixed payload (u64 size, then the bytes)
    std::string blob() { return bytes(size_t(get<uint64_t>())); }
    size_t left() const { return n_ - off_; }

private:
    void need(size_t k) const {
        if (k > n_ - off_) throw std::runtime_error("truncated archive");
    }
    const uint8_t* p_;
    size_t n_, off_ = 0;
};

std::string read_whole(const std::string& path) {
    std::ifstream in(path, std::ios::binary);
    if (!in) throw std::runtime_error("cannot open " + path);
    std::ostringstream ss;
    ss << in.rdbuf();
    return ss.str();
}

// fast-lzma2 stream -> bytes.
std::string fl2_decode(const std::string& src, int threads) {
    FL2_DStream* ds = FL2_createDStreamMt(unsigned(threads));
    if (!ds) throw std::runtime_error("fast-lzma2: cannot create a decoder");
    std::string out;
    try {
        size_t r = FL2_initDStream(ds);
        if (FL2_isError(r)) throw std::runtime_error(std::string("fast-lzma2: ") + FL2_getErrorName(r));
        FL2_inBuffer in = {src.data(), src.size(), 0};
        std::vector<char> buf(size_t(1) << 22);
        for (;;) {
            FL2_outBuffer ob = {buf.data(), buf.size(), 0};
            r = FL2_decompressStream(ds, &ob, &in);
            if (FL2_isError(r)) throw std::runtime_error(std::string("fast-lzma2: ") + FL2_getErrorName(r));
            out.append(buf.data(), ob.pos);
            if (r == 0) break;
            if (ob.pos == 0 && in.pos == in.size) throw std::runtime_error("fast-lzma2: truncated stream");
        }
    } catch (...) {
        FL2_freeDStream(ds);
        throw;
    }
    FL2_freeDStream(ds);
    return out;
}

template <class T>
std::vector<T> as_array(const std::string& bytes) {
    if (bytes.size() % sizeof(T)) throw std::runtime_error("stream size is not a whole number of values");
    std::vector<T> v(bytes.size() / sizeof(T));
    if (!v.empty()) std::memcpy(v.data(), bytes.data(), bytes.size());
    return v;
}

// ---- coded payloads (the formats LzmaLib.cpp writes), decoded without the
// wrappers' exit() paths

struct MemByteIn {
    IByteIn vt;
    const Byte* cur;
    const Byte* lim;
    bool overrun;
};
Byte mem_read_byte(const IByteIn* p) {
    MemByteIn* m = reinterpret_cast<MemByteIn*>(const_cast<IByteIn*>(p));
    if (m->cur < m->lim) return *m->cur++;
    m->overrun = true;
    return 0;
}

// LZMA: 5 property bytes, then the raw LZMA stream.
void lzma_payload(const uint8_t* src, size_t n, uint8_t* dst, size_t out) {
    if (n < LZMA_PROPS_SIZE) throw std::runtime_error("corrupt LZMA stream");
    SizeT dl = out, sl = n - LZMA_PROPS_SIZE;
    ELzmaStatus st;
    const SRes r = LzmaDecode(dst, &dl, src + LZMA_PROPS_SIZE, &sl, src, LZMA_PROPS_SIZE, LZMA_FINISH_ANY, &st,
                              &g_Alloc);
    if (r != SZ_OK || dl != out) throw std::runtime_error("corrupt LZMA stream");
}

// PPMd (variant H, 7z range coder): the model order, the model memory size
// (u32), then the range-coded symbols; every coded byte must be consumed.
void ppmd_payload(const uint8_t* src, size_t n, uint8_t* dst, size_t out) {
    if (n < 5) throw std::runtime_error("corrupt PPMd stream");
    const unsigned order = src[0];
    uint32_t mem;
    std::memcpy(&mem, src + 1, 4);
    if (order < PPMD7_MIN_ORDER || order > PPMD7_MAX_ORDER || mem < PPMD7_MIN_MEM_SIZE || mem > PPMD7_MAX_MEM_SIZE)
        throw std::runtime_error("corrupt PPMd stream properties");
    CPpmd7 ppmd;
    Ppmd7_Construct(&ppmd);
    if (!Ppmd7_Alloc(&ppmd, mem, &g_Alloc)) throw std::bad_alloc();
    Ppmd7_Init(&ppmd, order);
    MemByteIn in{{mem_read_byte}, src + 5, src + n, false};
    CPpmd7z_RangeDec rd;
    Ppmd7z_RangeDec_CreateVTable(&rd);
    rd.Stream = &in.vt;
    bool ok = Ppmd7z_RangeDec_Init(&rd) != 0;
    size_t i = 0;
    if (ok) {
        for (; i < out; ++i) {
            const int sym = Ppmd7_DecodeSymbol(&ppmd, &rd.vt);
            if (sym < 0 || in.overrun) break;
            dst[i] = Byte(sym);
        }
    }
    ok = ok && i == out && !in.overrun && in.cur == in.lim && Ppmd7z_RangeDec_IsFinishedOK(&rd);
    Ppmd7_Free(&ppmd, &g_Alloc);
    if (!ok) throw std::runtime_error("corrupt PPMd stream");
}

// PgRC's var-len DNA coding: a coder byte (static or dynamic book) and a book
// id, the code book as text (up to 256 codes of one to four symbols, one per
// line, the first a single symbol, ended by a zero byte), then one byte per
// code, each standing for its code's symbols.
void varlen_payload(const uint8_t* src, size_t n, uint8_t* dst, size_t out) {
    using VL = PgSAHelpers::VarLenDNACoder;
    if (n < 2 || (src[0] != VL::STATIC_CODES_CODER_PARAM && src[0] != VL::DYNAMIC_CODES_CODER_PARAM))
        throw std::runtime_error("corrupt var-len DNA stream");
    const uint8_t* book = src + 2;
    const uint8_t* end = static_cast<const uint8_t*>(std::memchr(book, 0, n - 2));
    if (!end) throw std::runtime_error("corrupt var-len DNA code book");
    std::vector<std::string> codes;
    const uint8_t* a = book;
    for (;;) {
        const uint8_t* b = static_cast<const uint8_t*>(std::memchr(a, '\n', size_t(end - a)));
        const uint8_t* e = b ? b : end;
        if (e - a > 4 || codes.size() == 256) throw std::runtime_error("corrupt var-len DNA code book");
        codes.emplace_back(reinterpret_cast<const char*>(a), size_t(e - a));
        if (!b) break;
        a = b + 1;
    }
    if (codes[0].size() != 1) throw std::runtime_error("corrupt var-len DNA code book");
    size_t o = 0;
    for (const uint8_t* p = end + 1; p < src + n; ++p) {
        if (*p >= codes.size()) continue;  // an unused code stands for nothing
        const std::string& c = codes[*p];
        if (c.size() > out - o) throw std::runtime_error("var-len DNA stream longer than stated");
        std::memcpy(dst + o, c.data(), c.size());
        o += c.size();
    }
    if (o != out) throw std::runtime_error("var-len DNA stream shorter than stated");
}

// A payload read front to back: size-prefixed blobs (u64 size, bytes) and
// the LZMA SDK containers of LzmaLib.cpp (decoded size, coded size, coder,
// coded bytes), which carry no size prefix of their own.  A container's
// header is checked here before its bytes go to the coder, which ends the
// process on the errors it detects itself.
class Cursor {
public:
    explicit Cursor(const std::string& s) : s_(s) {}
    std::string blob() {
        const uint64_t n = u64_at(off_);
        need(off_ + 8, n);
        std::string r = s_.substr(off_ + 8, size_t(n));
        off_ += 8 + size_t(n);
        return r;
    }
    template <class T>
    std::vector<T> values() {
        const std::string b = text();
        if (b.size() % sizeof(T)) throw std::runtime_error("coded stream size is not a whole number of values");
        std::vector<T> v(b.size() / sizeof(T));
        if (!v.empty()) std::memcpy(v.data(), b.data(), b.size());
        return v;
    }
    std::string text() {
        const size_t end = container_end(off_, 0);
        std::string v = decode_at(off_);
        off_ = end;
        return v;
    }
    bool done() const { return off_ == s_.size(); }

private:
    void need(size_t at, uint64_t k) const {
        if (at > s_.size() || k > s_.size() - at) throw std::runtime_error("truncated coded stream");
    }
    uint64_t u64_at(size_t at) const {
        need(at, 8);
        uint64_t v;
        std::memcpy(&v, s_.data() + at, 8);
        return v;
    }
    // end of the container at `at`, its header checked
    size_t container_end(size_t at, int depth) const {
        const uint64_t dest = u64_at(at);
        if (dest == 0) return at + 8;
        if (dest > (uint64_t(1) << 40)) throw std::runtime_error("implausible decoded size in a coded stream");
        const uint64_t src = u64_at(at + 8);
        need(at + 16, 1);
        const uint8_t coder = uint8_t(s_[at + 16]);
        if (coder == COMPOUND_CODER_TYPE) {
            // a VarLenDNACoder layer over an inner container of `src` bytes
            need(at + 17, 1);
            if (depth > 0 || uint8_t(s_[at + 17]) != VARLEN_DNA_CODER || u64_at(at + 18) != src)
                throw std::runtime_error("unsupported compound coded stream");
            return container_end(at + 18, depth + 1);
        }
        if (coder != LZMA_CODER && coder != PPMD7_CODER) throw std::runtime_error("unsupported coder in a coded stream");
        need(at + 17, src);
        return at + 17 + size_t(src);
    }
    // the decoded bytes of the (checked) container at `at`
    std::string decode_at(size_t at) const {
        const uint64_t dest = u64_at(at);
        std::string out(size_t(dest), '\0');
        if (dest == 0) return out;
        const uint64_t src = u64_at(at + 8);
        const uint8_t coder = uint8_t(s_[at + 16]);
        uint8_t* d = reinterpret_cast<uint8_t*>(&out[0]);
        if (coder == COMPOUND_CODER_TYPE) {
            const std::string inner = decode_at(at + 18);  // src bytes of var-len DNA coding
            varlen_payload(reinterpret_cast<const uint8_t*>(inner.data()), inner.size(), d, out.size());
            return out;
        }
        const uint8_t* p = reinterpret_cast<const uint8_t*>(s_.data()) + at + 17;
        if (coder == LZMA_CODER)
            lzma_payload(p, size_t(src), d, out.size());
        else
            ppmd_payload(p, size_t(src), d, out.size());
        return out;
    }
    const std::string& s_;
    size_t off_ = 0;
};

// The strand stream through the bsc executable (decompress.cu:301-317).
std::string bsc_decode(const std::string& bsc, const std::string& dir, const std::string& data, uint32_t block) {
    const std::string tag = std::to_string(getpid()) + "_" + std::to_string(block);
    const std::string in = dir + "/strand_" + tag + ".bsc", out = dir + "/strand_" + tag + ".txt";
    {
        std::ofstream f(in, std::ios::binary);
        f.write(data.data(), std::streamsize(data.size()));
        if (!f) throw std::ios_base::failure("cannot write " + in);
    }
    const std::string cmd = "'" + bsc + "' d '" + in + "' '" + out + "' > /dev/null";
    const int rc = std::system(cmd.c_str());
    std::remove(in.c_str());
    if (rc != 0) {
        std::remove(out.c_str());
        throw std::runtime_error("bsc failed: " + cmd);
    }
    std::string s = read_whole(out);
    std::remove(out.c_str());
    return s;
}

// The range decoder and adaptive frequency model of the mismatch-offset
// streams: the CLR range coder (32-bit range and code, 64-bit low, 2^24
// renormalisation threshold, eight start bytes of which the last four form the
// code) and a model of NSYM symbols kept roughly sorted by frequency (step 8,
// halved above 2^16 - 32, one neighbour swap every 16 symbols), as the
// encoder's vendored copies define them (range_coder/clr.cdr,
// range_coder/simple_model.h).  Restated here with two guards the originals
// lack, so a corrupt stream is an error and not an out-of-bounds read or a
// division by zero: the decoded frequency must lie below the model's total,
// and the range must stay at least the total.  Bytes past the stream read as
// zero.
class OffRangeDecoder {
public:
    OffRangeDecoder(const uint8_t* p, size_t n) : p_(p), end_(p + n) {
        for (int i = 0; i < 8; ++i) code_ = (code_ << 8) | next();
    }
    uint32_t get_freq(uint32_t tot) {
        range_ /= tot;
        if (range_ == 0) throw std::runtime_error("corrupt mismatch offset stream");
        return code_ / range_;
    }
    void decode(uint32_t cum, uint32_t freq) {
        const uint32_t t = cum * range_;
        low_ += t;
        code_ -= t;
        range_ *= freq;
        while (range_ < (1u << 24)) {
            if (uint8_t((low_ ^ (low_ + range_)) >> 56)) range_ = (uint32_t(low_) | ((1u << 24) - 1)) - uint32_t(low_);
            code_ = (code_ << 8) | next();
            range_ <<= 8;
            low_ <<= 8;
        }
    }

private:
    uint32_t next() { return p_ < end_ ? *p_++ : 0u; }
    const uint8_t* p_;
    const uint8_t* end_;
    uint64_t low_ = 0;
    uint32_t range_ = 0xFFFFFFFFu, code_ = 0;
};

template <int NSYM>
class OffModel {
public:
    OffModel() {
        for (int i = 0; i < NSYM; ++i) {
            sym_[i] = uint16_t(i);
            freq_[i] = 1;
        }
    }
    uint16_t decode(OffRangeDecoder& rc) {
        const uint32_t f = rc.get_freq(tot_);
        if (f >= tot_) throw std::runtime_error("corrupt mismatch offset stream");
        uint32_t acc = 0;
        int i = 0;
        while (acc + freq_[i] <= f) acc += freq_[i++];  // ends below NSYM since f < tot_
        rc.decode(acc, freq_[i]);
        freq_[i] = uint16_t(freq_[i] + STEP);
        tot_ += STEP;
        if (tot_ > MAXF) {
            tot_ = 0;
            for (int k = 0; k < NSYM; ++k) {
                freq_[k] = uint16_t(freq_[k] - (freq_[k] >> 1));
                tot_ += freq_[k];
            }
        }
        const uint16_t out = sym_[i];
        if (((++bub_ & 15u) == 0) && i > 0 && freq_[i] > freq_[i - 1]) {
            std::swap(freq_[i], freq_[i - 1]);
            std::swap(sym_[i], sym_[i - 1]);
        }
        return out;
    }

private:
    static constexpr uint32_t STEP = 8, MAXF = (1u << 16) - 32;
    uint16_t sym_[NSYM], freq_[NSYM];
    uint32_t tot_ = NSYM, bub_ = 0;
};

// Mismatch offsets of the records with m mismatches, from their range-coded
// stream: the inverse of the encoder's flag / first / gap coding
// (decompress.cu:357-416): `m` offsets for each of `records` records.
template <size_t MaxL>
std::vector<uint16_t> offsets_decode(const std::string& coded, size_t m, size_t records, int L) {
    OffRangeDecoder rc(reinterpret_cast<const uint8_t*>(coded.data()), coded.size());
    OffModel<2> flag;
    OffModel<int(MaxL / 2 + 1)> first;
    OffModel<int(MaxL)> value;
    std::vector<uint16_t> out(records * m);
    for (size_t r = 0; r < records; ++r) {
        uint16_t* t = out.data() + r * m;
        const bool from_end = flag.decode(rc) != 0;
        if (!from_end) {
            // first offset, then gaps forward
            t[0] = first.decode(rc);
            if (m == 2) {
                t[1] = uint16_t(value.decode(rc) + t[0] + 1);
            } else if (m > 2) {
                const uint32_t min_gap = value.decode(rc) + 1u;
                for (size_t k = 1; k < m; ++k) t[k] = uint16_t(value.decode(rc) + t[k - 1] + min_gap);
            }
        } else {
            // last offset from the read's end, then gaps backward
            t[m - 1] = uint16_t(L - 1 - first.decode(rc));
            if (m == 2) {
                t[0] = uint16_t(t[1] - value.decode(rc) - 1);
            } else if (m > 2) {
                const uint32_t min_gap = value.decode(rc) + 1u;
                for (size_t k = m - 1; k > 0; --k) t[k - 1] = uint16_t(t[k] - value.decode(rc) - min_gap);
            }
        }
    }
    return out;
}

std::vector<uint16_t> offsets_for(int L, const std::string& coded, size_t m, size_t records) {
    if (L <= 128) return offsets_decode<128>(coded, m, records, L);
    if (L <= 256) return offsets_decode<256>(coded, m, records, L);
    if (L <= 384) return offsets_decode<384>(coded, m, records, L);
    return offsets_decode<512>(coded, m, records, L);
}

// Base-128 little-endian integer, high bit set on every byte but the last.
uint64_t read_frugal(const std::string& s, size_t& pos) {
    uint64_t v = 0, scale = 1;
    for (;;) {
        if (pos >= s.size()) throw std::runtime_error("truncated repeat map");
        const uint8_t b = uint8_t(s[pos++]);
        v += scale * (b & 127u);
        scale *= 128;
        if (b < 128) break;
    }
    return v;
}

char complement(char b) {
    switch (b) {
        case 'A': return 'T';
        case 'T': return 'A';
        case 'C': return 'G';
        case 'G': return 'C';
        case 'a': return 't';
        case 't': return 'a';
        case 'c': return 'g';
        case 'g': return 'c';
        default: return 'N';
    }
}

// Repeats removed by the RefMatcher put back (recoverRef, decompress.cu:
// 417-443): each '%' in `coded` stands for the reverse complement of a
// stretch of the source (the text recovered so far when self_source, else
// `src`), at the offset of the next entry of `offs` (u32 or u64) and with
// the length of the next entry of `lens` plus the stream's base length.
std::string recover_ref(const std::string& coded, const std::string* src, const std::string& offs,
                        const std::string& lens, bool off32) {
    std::string out;
    out.reserve(coded.size());
    size_t lp = 0, op = 0;
    // an empty length stream (no repeat was removed) reads as base length 0
    const uint64_t base_len = lens.empty() ? 0 : read_frugal(lens, lp);
    size_t at = 0;
    for (;;) {
        const size_t mark = coded.find('%', at);
        if (mark == std::string::npos) break;
        out.append(coded, at, mark - at);
        at = mark + 1;
        uint64_t sp;
        if (off32) {
            if (op + 4 > offs.size()) throw std::runtime_error("truncated repeat offsets");
            uint32_t v;
            std::memcpy(&v, offs.data() + op, 4);
            sp = v;
            op += 4;
        } else {
            if (op + 8 > offs.size()) throw std::runtime_error("truncated repeat offsets");
            std::memcpy(&sp, offs.data() + op, 8);
            op += 8;
        }
        const uint64_t len = read_frugal(lens, lp) + base_len;
        const std::string& s = src ? *src : out;
        if (sp > s.size() || len > s.size() - sp) throw std::runtime_error("repeat outside its source");
        const size_t o = out.size();
        out.resize(o + len);
        for (uint64_t k = 0; k < len; ++k) out[o + k] = complement(s[sp + len - 1 - k]);
    }
    out.append(coded, at, std::string::npos);
    return out;
}

// Positions of paired-end reads in preserved order from the pair coder
// (extract_id_to_pos, decompress.cu:115-216): the first mate's position
// directly; the second's as a 16-bit offset from it, or a 16-bit change of
// the last large offset, or verbatim; pairs visited in order of their first
// mate's position.
template <class T>
std::vector<uint64_t> pe_positions(const std::string& payload, uint32_t reads, int threads) {
    Cursor r(payload);
    const std::vector<T> first = as_array<T>(fl2_decode(r.blob(), threads));
    const auto off_flag = r.values<uint8_t>();
    const auto off_first = r.values<uint8_t>();
    const auto off_val = r.values<uint16_t>();
    const auto d_flag = r.values<uint8_t>();
    const auto d_first = r.values<uint8_t>();
    const auto d_val = r.values<int16_t>();
    const std::vector<T> verbatim = as_array<T>(fl2_decode(r.blob(), threads));
    if (!r.done()) throw std::runtime_error("bytes after the pair position streams");
    const uint32_t pairs = reads / 2;
    if (first.size() != pairs || off_flag.size() != pairs) throw std::runtime_error("pair position streams disagree");
    // pairs by their first mate's position, ties in pair order
    const std::vector<uint32_t> order = stable_order(first.data(), first.size(), threads);
    std::vector<uint64_t> second(pairs);
    size_t io = 0, idf = 0, idv = 0, iv = 0;
    int64_t ref_prev = 0, prev = 0;
    bool match = false;
    auto at = [](const auto& v, size_t i) {
        if (i >= v.size()) throw std::runtime_error("pair position streams too short");
        return v[i];
    };
    for (uint32_t q = 0; q < pairs; ++q) {
        const uint32_t p = order[q];
        const int64_t base = int64_t(first[p]);
        int64_t pos;
        if (off_flag[q]) {
            const int64_t rel = at(off_val, io);
            pos = at(off_first, io) ? base + rel : base - rel;
            ++io;
        } else if (at(d_flag, idf++)) {
            const int64_t rel = ref_prev + at(d_val, idv);
            ref_prev = rel;
            prev = rel;
            pos = at(d_first, idv) ? base + rel : base - rel;
            ++idv;
            match = true;
        } else {
            pos = int64_t(at(verbatim, iv++));
            const int64_t rel = pos > base ? pos - base : base - pos;
            if (!match || ref_prev != prev) ref_prev = rel;
            match = false;
            prev = rel;
        }
        second[p] = uint64_t(pos);
    }
    std::vector<uint64_t> out(size_t(pairs) * 2);
    for (uint32_t p = 0; p < pairs; ++p) {
        out[2 * size_t(p)] = uint64_t(first[p]);
        out[2 * size_t(p) + 1] = second[p];
    }
    return out;
}

// Output order of paired-end reads without preserved order
// (extract_pe_pair_order, decompress.cu:219-299): walking the records in
// pseudogenome order, each record not yet placed opens a pair whose other
// record lies an offset further (8-bit, an 8-bit change of the last large
// offset, or verbatim); then a flag per pair tells whether the mates swap.
std::vector<uint32_t> pe_order_decode(const std::string& payload, uint32_t reads, int threads) {
    Cursor r(payload);
    const auto off8_flag = r.values<uint8_t>();
    const auto off8_val = r.values<uint8_t>();
    const auto d8_flag = r.values<uint8_t>();
    const auto off_swap = r.values<uint8_t>();
    const auto far_swap = r.values<uint8_t>();
    const auto d8_val = as_array<int8_t>(fl2_decode(r.blob(), threads));
    const auto far = as_array<uint32_t>(fl2_decode(r.blob(), threads));
    if (!r.done()) throw std::runtime_error("bytes after the pair order streams");
    auto at = [](const auto& v, size_t i) {
        if (i >= v.size()) throw std::runtime_error("pair order streams too short");
        return v[i];
    };
    std::vector<uint32_t> order(reads);
    std::vector<uint8_t> placed(reads, 0);
    size_t pair = 0, iv = 0, idf = 0, idv = 0, ifar = 0;
    int64_t ref_prev = 0, prev = 0;
    bool match = false;
    for (uint32_t i = 0; i < reads; ++i) {
        if (placed[i]) continue;
        int64_t d;
        if (at(off8_flag, pair)) {
            d = at(off8_val, iv++);
        } else if (at(d8_flag, idf++)) {
            d = ref_prev + at(d8_val, idv++);
            ref_prev = d;
            prev = d;
            match = true;
        } else {
            d = int64_t(at(far, ifar++));
            if (!match || ref_prev != prev) ref_prev = d;
            match = false;
            prev = d;
        }
        const int64_t j = int64_t(i) + d;
        if (2 * pair + 1 >= reads || d <= 0 || j >= int64_t(reads) || placed[size_t(j)])
            throw std::runtime_error("pair order stream is inconsistent");
        order[2 * pair] = i;
        order[2 * pair + 1] = uint32_t(j);
        placed[size_t(j)] = 1;
        ++pair;
    }
    size_t is = 0, ifs = 0;
    for (size_t p = 0; p < reads / 2; ++p) {
        const bool swap = off8_flag[p] ? at(off_swap, is++) : at(far_swap, ifs++);
        if (swap) std::swap(order[2 * p], order[2 * p + 1]);
    }
    return order;
}

// Cumulative read positions from a read-offset stream (decompress.cu:67-82);
// the unmapped streams hold read_len minus the step.
void positions_from_offsets(const std::vector<uint16_t>& steps, int L, bool complemented, uint64_t* pos) {
    uint64_t p = 0;
    for (size_t i = 0; i < steps.size(); ++i) {
        const uint64_t st = complemented ? uint64_t(uint16_t(L - steps[i])) : steps[i];
        p = i == 0 ? st : p + st;
        pos[i] = p;
    }
}

struct Block {
    uint32_t reads = 0;
    char table[128][4];
    bool join32 = false, ref32 = false;
    uint64_t ref_size = 0, unmap_size = 0, unmap_n_size = 0;
    std::string strand, hq, lq, nq, mis_base;
    std::vector<uint8_t> mis_cnt;
    std::vector<uint64_t> mis_first;  // first offset / base index of each record
    std::vector<uint16_t> mis_off;
    std::vector<uint64_t> pos;       // no preserved order: per record (hq, lq, N)
    size_t hq_n = 0, lq_n = 0;       // no preserved order: hq and lq record counts
    std::vector<uint32_t> pe_order;  // no preserved order, paired-end: output -> record
    std::vector<uint64_t> id_pos;    // preserved order: per read
};

// One block's fields and coded payloads, in archive order (the block layout
// of compress.cu:1364-2146, read back at decompress.cu:763-814).
struct BlockPayloads {
    uint32_t reads = 0;
    char table[16];
    bool join32 = false, ref32 = false;
    uint64_t ref_size = 0, unmap_size = 0, unmap_n_size = 0;
    std::string idpos, strand, ref, roff, unoff, uoff, peorder, maps[6], cnt, base;
    int max_mm = 0;
    std::vector<std::string> off;  // index m = 1 .. max_mm
};

BlockPayloads read_block(Reader& ar, bool po, bool pe) {
    BlockPayloads b;
    b.reads = ar.get<uint32_t>();
    const std::string t = ar.bytes(16);
    std::memcpy(b.table, t.data(), 16);
    if (po) b.join32 = ar.get<uint8_t>() != 0;
    b.ref32 = ar.get<uint8_t>() != 0;
    b.ref_size = ar.get<uint64_t>();
    b.unmap_size = ar.get<uint64_t>();
    b.unmap_n_size = ar.get<uint64_t>();
    if (po) b.idpos = ar.blob();
    b.strand = ar.blob();
    b.ref = ar.blob();
    if (!po) {
        b.roff = ar.blob();
        b.unoff = ar.blob();
        b.uoff = ar.blob();
        if (pe) b.peorder = ar.blob();
    }
    for (auto& m : b.maps) m = ar.blob();
    b.cnt = ar.blob();
    b.base = ar.blob();
    b.max_mm = ar.get<uint8_t>();
    b.off.resize(size_t(b.max_mm) + 1);
    for (int m = 1; m <= b.max_mm; ++m) b.off[size_t(m)] = ar.blob();
    return b;
}

// Mismatch offsets and symbols of a learned block: the container (u64 base
// count, u64 payload length, u8 LEARNED_CODER) holds u32 model size, the
// model and the stream; records are the main-pseudogenome reads in record
// order (read id order with preserved order), with their positions and
// strands already decoded.  Bases become the symbols the plain stream
// would hold: their rank in the block's decoder table row.
void learned_mismatches(Block& b, const std::string& payload, bool po, int L) {
    if (payload.size() < 21) throw std::runtime_error("learned container too short");
    uint64_t nbase, clen;
    uint32_t msize;
    std::memcpy(&nbase, payload.data(), 8);
    std::memcpy(&clen, payload.data() + 8, 8);
    std::memcpy(&msize, payload.data() + 17, 4);
    if (clen != payload.size() - 17 || msize != sizeof(learned::Model) || clen < 4ull + msize)
        throw std::runtime_error("learned container is malformed");
    learned::Model M;
    std::memcpy(&M, payload.data() + 21, sizeof(M));
    const uint8_t* stream = reinterpret_cast<const uint8_t*>(payload.data()) + 21 + msize;
    const size_t sbytes = size_t(clen - 4 - msize);
    const size_t R = b.mis_cnt.size();
    if (b.mis_first[R] != nbase) throw std::runtime_error("learned container: base count disagrees with the counts");
    std::vector<uint64_t> pos;
    pos.reserve(R);
    if (po) {
        for (uint64_t p : b.id_pos)
            if (p < b.hq.size()) pos.push_back(p);
    } else {
        if (b.hq_n != R) throw std::runtime_error("record streams disagree");
        pos.assign(b.pos.begin(), b.pos.begin() + R);
    }
    if (pos.size() != R || b.strand.size() != R) throw std::runtime_error("record streams disagree");
    std::vector<uint8_t> strand(R);
    for (size_t r = 0; r < R; ++r) strand[r] = b.strand[r] == '1';
    b.mis_off.assign(nbase, 0);
    std::string bases(nbase, '\0');
    const std::string why =
        learned::decode_stream(M, stream, sbytes, reinterpret_cast<const uint8_t*>(b.hq.data()), b.hq.size(), L, R,
                               pos.data(), strand.data(), b.mis_cnt.data(), b.mis_off.data(), &bases[0]);
    if (!why.empty()) throw std::runtime_error(why);
    b.mis_base.assign(nbase, '\0');
    for (size_t r = 0; r < R; ++r)
        for (uint64_t k = b.mis_first[r]; k < b.mis_first[r + 1]; ++k) {
            const char gb = b.hq[pos[r] + b.mis_off[k]];
            int sym = -1;
            for (int j = 0; j < 4; ++j)
                if (b.table[uint8_t(gb) & 127][j] == bases[k]) sym = j;
            if (sym < 0) throw std::runtime_error("learned stream: base outside the decoder table");
            b.mis_base[k] = char(sym);
        }
}

Block decode_block(Reader& ar, bool po, bool pe, int L, const DecodeParams& dp, uint32_t index) {
    Block b;
    BlockPayloads bp = read_block(ar, po, pe);
    b.reads = bp.reads;
    std::memset(b.table, 'N', sizeof(b.table));
    const char rows[4] = {'A', 'T', 'C', 'G'};
    for (int r = 0; r < 4; ++r) std::memcpy(b.table[int(rows[r])], bp.table + 4 * r, 4);
    b.join32 = bp.join32;
    b.ref32 = bp.ref32;
    b.ref_size = bp.ref_size;
    b.unmap_size = bp.unmap_size;
    b.unmap_n_size = bp.unmap_n_size;
    const std::string &s_idpos = bp.idpos, &s_strand = bp.strand, &s_ref = bp.ref, &s_roff = bp.roff,
                      &s_unoff = bp.unoff, &s_uoff = bp.uoff, &s_peorder = bp.peorder, &s_cnt = bp.cnt,
                      &s_base = bp.base;
    const std::string* maps = bp.maps;
    const int max_mm = bp.max_mm;
    const std::vector<std::string>& s_off = bp.off;

    const int thr = dp.threads;
    auto f_strand = std::async(std::launch::async, [&] { return bsc_decode(dp.bsc_path, dp.tmpdir, s_strand, index); });
    auto f_ref = std::async(std::launch::async, [&] {
        const std::string packed = fl2_decode(s_ref, thr);
        std::string ref(size_t(b.ref_size + b.unmap_size + b.unmap_n_size), '\0');
        if (!ref.empty())
            varlen_payload(reinterpret_cast<const uint8_t*>(packed.data()), packed.size(),
                           reinterpret_cast<uint8_t*>(&ref[0]), ref.size());
        return ref;
    });
    std::future<std::string> f_maps[6];
    for (int k = 0; k < 6; ++k)
        f_maps[k] = std::async(std::launch::async, [&, k] { return Cursor(maps[k]).text(); });
    // a block whose mismatch bases and offsets the learned coder wrote: the
    // base container carries LEARNED_CODER, the model and the stream, and
    // is decoded below once positions and pseudogenome are known
    const bool learned = s_base.size() >= 17 && uint8_t(s_base[16]) == LEARNED_CODER;
    auto f_base = std::async(std::launch::async, [&] { return learned ? std::string() : Cursor(s_base).text(); });
    auto f_mis = std::async(std::launch::async, [&] {
        b.mis_cnt = Cursor(s_cnt).values<uint8_t>();
        const size_t R = b.mis_cnt.size();
        b.mis_first.resize(R + 1);
        std::vector<size_t> per(size_t(max_mm) + 1, 0);
        uint64_t acc = 0;
        for (size_t r = 0; r < R; ++r) {
            b.mis_first[r] = acc;
            acc += b.mis_cnt[r];
            if (b.mis_cnt[r] > max_mm) throw std::runtime_error("mismatch count above the block's maximum");
            ++per[b.mis_cnt[r]];
        }
        b.mis_first[R] = acc;
        if (learned) return;  // offsets come from the learned stream
        // every class decodes on its own; then records take their offsets in order
        std::vector<std::future<std::vector<uint16_t>>> f(size_t(max_mm) + 1);
        for (int m = 1; m <= max_mm; ++m)
            f[size_t(m)] = std::async(std::launch::async, [&, m] {
                return offsets_for(L, s_off[size_t(m)], size_t(m), per[size_t(m)]);
            });
        std::vector<std::vector<uint16_t>> cls(size_t(max_mm) + 1);
        for (int m = 1; m <= max_mm; ++m) cls[size_t(m)] = f[size_t(m)].get();
        b.mis_off.resize(acc);
        std::vector<size_t> next(size_t(max_mm) + 1, 0);
        for (size_t r = 0; r < R; ++r) {
            const int m = b.mis_cnt[r];
            if (!m) continue;
            std::memcpy(b.mis_off.data() + b.mis_first[r], cls[size_t(m)].data() + next[size_t(m)], size_t(m) * 2);
            next[size_t(m)] += size_t(m);
        }
    });
    std::future<void> f_pos;
    if (!po) {
        f_pos = std::async(std::launch::async, [&] {
            const auto hq = Cursor(s_roff).values<uint16_t>();
            const auto lq = Cursor(s_uoff).values<uint16_t>();
            const auto nq = Cursor(s_unoff).values<uint16_t>();
            if (hq.size() + lq.size() + nq.size() != b.reads)
                throw std::runtime_error("read offsets disagree with the block's read count");
            b.pos.resize(b.reads);
            positions_from_offsets(hq, L, false, b.pos.data());
            positions_from_offsets(lq, L, true, b.pos.data() + hq.size());
            positions_from_offsets(nq, L, true, b.pos.data() + hq.size() + lq.size());
            b.hq_n = hq.size();
            b.lq_n = lq.size();
        });
    }
    std::future<void> f_order;
    if (!po && pe) f_order = std::async(std::launch::async, [&] { b.pe_order = pe_order_decode(s_peorder, b.reads, thr); });
    std::future<void> f_idpos;
    if (po) {
        f_idpos = std::async(std::launch::async, [&] {
            if (!pe) {
                const std::string raw = fl2_decode(s_idpos, thr);
                if (b.join32) {
                    const auto v = as_array<uint32_t>(raw);
                    b.id_pos.assign(v.begin(), v.end());
                } else {
                    b.id_pos = as_array<uint64_t>(raw);
                }
            } else {
                b.id_pos = b.join32 ? pe_positions<uint32_t>(s_idpos, b.reads, thr)
                                    : pe_positions<uint64_t>(s_idpos, b.reads, thr);
            }
            if (b.id_pos.size() != b.reads) throw std::runtime_error("read positions disagree with the read count");
        });
    }
    // collect every task before rethrowing any error (they use this frame)
    std::exception_ptr err;
    auto join = [&](auto& f) {
        try {
            if (f.valid()) f.get();
        } catch (...) {
            if (!err) err = std::current_exception();
        }
    };
    std::string ref, mapv[6];
    try {
        b.strand = f_strand.get();
    } catch (...) {
        if (!err) err = std::current_exception();
    }
    try {
        ref = f_ref.get();
    } catch (...) {
        if (!err) err = std::current_exception();
    }
    for (int k = 0; k < 6; ++k) try {
            mapv[k] = f_maps[k].get();
        } catch (...) {
            if (!err) err = std::current_exception();
        }
    try {
        b.mis_base = f_base.get();
    } catch (...) {
        if (!err) err = std::current_exception();
    }
    join(f_mis);
    join(f_pos);
    join(f_order);
    join(f_idpos);
    if (err) std::rethrow_exception(err);

    // the three pseudogenomes, repeats put back (decompress.cu:915-927)
    const std::string hq_coded = ref.substr(0, size_t(b.ref_size));
    const std::string lq_coded = ref.substr(size_t(b.ref_size), size_t(b.unmap_size));
    const std::string nq_coded = ref.substr(size_t(b.ref_size + b.unmap_size));
    b.hq = recover_ref(hq_coded, nullptr, mapv[0], mapv[1], b.ref32);
    b.lq = recover_ref(lq_coded, &b.hq, mapv[2], mapv[3], b.ref32);
    b.nq = recover_ref(nq_coded, &b.hq, mapv[4], mapv[5], b.ref32);
    if (learned) learned_mismatches(b, s_base, po, L);
    if (b.strand.size() != b.mis_cnt.size() || b.mis_base.size() != b.mis_off.size())
        throw std::runtime_error("record streams disagree");
    return b;
}

// One read into dst (L bytes): a copy of its pseudogenome stretch; for a
// record of the main pseudogenome its mismatches patched in, then reverse
// complemented when its strand is '1' (decompress.cu:1000-1035).
inline void rebuild(const Block& b, int L, int kind, uint64_t p, size_t rec, char* dst) {
    const std::string& g = kind == 0 ? b.hq : kind == 1 ? b.lq : b.nq;
    if (p > g.size() || uint64_t(L) > g.size() - p) throw std::runtime_error("read outside its pseudogenome");
    std::memcpy(dst, g.data() + p, size_t(L));
    if (kind != 0) return;
    if (rec >= b.mis_cnt.size()) throw std::runtime_error("record index outside the record streams");
    const uint64_t f = b.mis_first[rec];
    for (uint32_t k = 0; k < b.mis_cnt[rec]; ++k) {
        const uint16_t o = b.mis_off[f + k];
        if (o >= L) throw std::runtime_error("mismatch offset outside the read");
        const uint8_t sym = uint8_t(b.mis_base[f + k]);
        if (sym > 3) throw std::runtime_error("bad mismatch symbol");
        dst[o] = b.table[uint8_t(dst[o]) & 127][sym];
    }
    if (b.strand[rec] == '1') {
        std::reverse(dst, dst + L);
        for (int k = 0; k < L; ++k) dst[k] = complement(dst[k]);
    }
}

// Writes the block's reads in the reference decoder's order: record order
// (or the pair order) without preserved order, read id order with it.
void write_block(const Block& b, bool po, bool pe, int L, std::ofstream& o1, std::ofstream& o2, int threads) {
    const size_t n = b.reads;
    // preserved order: the record of each main-pseudogenome read
    std::vector<uint64_t> rec_of;
    if (po) {
        rec_of.resize(n);
        uint64_t r = 0;
        for (size_t i = 0; i < n; ++i) {
            rec_of[i] = r;
            if (b.id_pos[i] < b.hq.size()) ++r;
        }
    }
    const size_t line = size_t(L) + 1;
    const size_t chunk = std::max<size_t>(2, ((size_t(64) << 20) / line) & ~size_t(1));
    std::vector<char> buf(std::min(n, chunk) * line);
    std::atomic<bool> bad{false};
    std::string why;
    for (size_t c0 = 0; c0 < n; c0 += chunk) {
        const size_t cn = std::min(chunk, n - c0);
#pragma omp parallel for num_threads(threads) schedule(static)
        for (size_t i = 0; i < cn; ++i) {
            if (bad.load(std::memory_order_relaxed)) continue;
            try {
                const size_t out = c0 + i;
                int kind;
                uint64_t p;
                size_t rec;
                if (po) {
                    const uint64_t q = b.id_pos[out];
                    rec = size_t(rec_of[out]);
                    if (q < b.hq.size()) {
                        kind = 0;
                        p = q;
                    } else if (q < b.hq.size() + b.lq.size()) {
                        kind = 1;
                        p = q - b.hq.size();
                    } else {
                        kind = 2;
                        p = q - b.hq.size() - b.lq.size();
                    }
                } else {
                    rec = pe ? b.pe_order[out] : out;
                    if (rec >= n) throw std::runtime_error("pair order outside the block");
                    p = b.pos[rec];
                    kind = rec < b.hq_n ? 0 : rec < b.hq_n + b.lq_n ? 1 : 2;
                }
                char* dst = buf.data() + i * line;
                rebuild(b, L, kind, p, rec, dst);
                dst[L] = '\n';
            } catch (const std::exception& e) {
#pragma omp critical
                if (!bad.exchange(true)) why = e.what();
            }
        }
        if (bad) throw std::runtime_error(why);
        if (!pe) {
            o1.write(buf.data(), std::streamsize(cn * line));
        } else {
            // even outputs to the first file, odd to the second
            for (size_t i = 0; i < cn; ++i) ((c0 + i) % 2 ? o2 : o1).write(buf.data() + i * line, std::streamsize(line));
        }
    }
}

}  // namespace

std::string learned_decode(const void* model, const uint8_t* p, size_t bytes, const uint8_t* ref, uint64_t rl, int L,
                           size_t records, const uint64_t* pos, const uint8_t* strand, const uint8_t* cnt,
                           uint16_t* off, char* base) {
    learned::Model M;
    std::memcpy(&M, model, sizeof(M));
    return learned::decode_stream(M, p, bytes, ref, rl, L, records, pos, strand, cnt, off, base);
}

ArchiveInfo archive_info(const std::string& archive) {
    const std::string data = read_whole(archive);
    Reader ar(data);
    ArchiveInfo info;
    info.preserve_order = ar.get<uint8_t>() != 0;
    info.paired_end = ar.get<uint8_t>() != 0;
    info.read_len = ar.get<uint16_t>();
    const int blocks = ar.get<uint8_t>();
    for (int k = 0; k < blocks; ++k) {
        const size_t before = ar.left();
        const BlockPayloads bp = read_block(ar, info.preserve_order, info.paired_end);
        info.block_reads.push_back(bp.reads);
        info.block_bytes.push_back(before - ar.left());
    }
    if (ar.left() != 0) throw std::runtime_error("bytes after the last block");
    return info;
}

DecodeResult decode_archive(const std::string& archive, const std::string& out_prefix, const DecodeParams& dp) {
    const std::string data = read_whole(archive);
    Reader ar(data);
    const bool po = ar.get<uint8_t>() != 0, pe = ar.get<uint8_t>() != 0;
    const int L = ar.get<uint16_t>();
    const int blocks = ar.get<uint8_t>();
    if (L < 1 || L > 511) throw std::runtime_error("read length in the archive header is out of range");
    DecodeResult res;
    res.read_len = L;
    res.paired_end = pe;
    res.preserve_order = po;
    std::ofstream o1, o2;
    const std::string f1 = out_prefix + (pe ? "_1.seq" : ".seq");
    o1.open(f1, std::ios::binary);
    if (!o1) throw std::ios_base::failure("cannot write " + f1);
    if (pe) {
        const std::string f2 = out_prefix + "_2.seq";
        o2.open(f2, std::ios::binary);
        if (!o2) throw std::ios_base::failure("cannot write " + f2);
    }
    DecodeParams p = dp;
    if (p.threads <= 0) p.threads = omp_get_max_threads();
    for (int k = 0; k < blocks; ++k) {
        const Block b = decode_block(ar, po, pe, L, p, uint32_t(k));
        if (pe && b.reads % 2) throw std::runtime_error("odd read count in a paired-end block");
        write_block(b, po, pe, L, o1, o2, p.threads);
        res.reads += b.reads;
        ++res.blocks;
    }
    if (ar.left() != 0) throw std::runtime_error("bytes after the last block");
    o1.flush();
    if (pe) o2.flush();
    if (!o1 || (pe && !o2)) throw std::ios_base::failure("cannot write the decoded reads");
    return res;
}

}  // namespace host
}  // namespace curc

namespace curc {
std::string& ctxless_error();
}

extern "C" int curc_decompress_file(const char* archive_path, const char* out_prefix, const char* bsc_path,
                                    const char* tmpdir, int threads, uint64_t* reads_out) {
    if (!archive_path || !out_prefix || !bsc_path || !tmpdir || threads < 0) {
        curc::ctxless_error() = "curc_decompress_file: null path or negative thread count";
        return CURC_ERR_ARG;
    }
    try {
        struct stat st;
        if (stat(archive_path, &st) != 0) throw std::ios_base::failure(std::string("cannot open ") + archive_path);
        curc::host::DecodeParams p;
        p.bsc_path = bsc_path;
        p.tmpdir = tmpdir;
        p.threads = threads;
        const auto r = curc::host::decode_archive(archive_path, out_prefix, p);
        if (reads_out) *reads_out = r.reads;
        return CURC_OK;
    } catch (const std::ios_base::failure& e) {
        curc::ctxless_error() = e.what();
        return CURC_ERR_IO;
    } catch (const std::exception& e) {
        curc::ctxless_error() = e.what();
        return CURC_ERR_STATE;
    }
}

extern "C" int curc_archive_info(const char* archive_path, int* preserve_order, int* paired_end, uint16_t* read_len,
                                 uint32_t* blocks, uint64_t* block_bytes, uint32_t* block_reads) {
    if (!archive_path) {
        curc::ctxless_error() = "curc_archive_info: null path";
        return CURC_ERR_ARG;
    }
    try {
        struct stat st;
        if (stat(archive_path, &st) != 0) throw std::ios_base::failure(std::string("cannot open ") + archive_path);
        const auto info = curc::host::archive_info(archive_path);
        if (preserve_order) *preserve_order = info.preserve_order;
        if (paired_end) *paired_end = info.paired_end;
        if (read_len) *read_len = uint16_t(info.read_len);
        if (blocks) *blocks = uint32_t(info.block_bytes.size());
        for (size_t k = 0; k < info.block_bytes.size(); ++k) {
            if (block_bytes) block_bytes[k] = info.block_bytes[k];
            if (block_reads) block_reads[k] = info.block_reads[k];
        }
        return CURC_OK;
    } catch (const std::ios_base::failure& e) {
        curc::ctxless_error() = e.what();
        return CURC_ERR_IO;
    } catch (const std::exception& e) {
        curc::ctxless_error() = e.what();
        return CURC_ERR_STATE;
    }
}
