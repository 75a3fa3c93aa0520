// CPU oracle for the CURC pseudogenome path -- TEST INFRASTRUCTURE ONLY.
//
// FASTQ ingest + block split (preprocess.cpp:66-283), block stream coding
// and archive layout (compress.cu:1911-2146), and a C API for the tests.
// The entropy coders are the reference's vendored third-party libraries,
// linked from oracle/_ref/libcurc_coders.a; the strand stream goes through
// the reference's `bsc` executable exactly as compress.cu does (util.cuh:527).
#include <sys/stat.h>
#include <unistd.h>

#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "oracle.hpp"

#ifndef ABS
#define ABS std::abs
#endif
#include <lzma/VarLenDNACoder/LzmaLib.h>
#include <range_coder/clr.cdr>
#include <range_coder/simple_model.h>

namespace lzma2 {
void lzma2_compress(const char* infile, const char* outfile, int level, int thread_num);
}

namespace oracle {
namespace {

std::string read_file(const std::string& path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("cannot open " + path);
    std::stringstream ss;
    ss << f.rdbuf();
    return ss.str();
}

void write_file(const std::string& path, const void* data, size_t n) {
    std::ofstream f(path, std::ios::binary);
    if (n) f.write(static_cast<const char*>(data), n);
}

template <size_t MaxL>
std::string offsets_coded(const std::vector<uint16_t>& a, size_t m) {
    // util.cuh:307-343: CLR range coder, adaptive flag/first/value models
    std::vector<char> buf(a.size() * sizeof(uint16_t) + 1024);
    RangeCoder rc{};
    rc.output(buf.data());
    rc.StartEncode();
    SIMPLE_MODEL<2> flag;
    SIMPLE_MODEL<MaxL / 2 + 1> first;
    SIMPLE_MODEL<MaxL> value;
    size_t i = 0;
    while (i < a.size()) {
        flag.encodeSymbol(&rc, a[i++]);
        first.encodeSymbol(&rc, a[i++]);
        if (m > 1) {
            if (m == 2) {
                value.encodeSymbol(&rc, a[i++]);
            } else {
                value.encodeSymbol(&rc, a[i++]);
                for (size_t k = 1; k < m; ++k) value.encodeSymbol(&rc, a[i++]);
            }
        }
    }
    rc.FinishEncode();
    return std::string(buf.data(), rc.size_out());
}

std::string offsets_for(int L, const std::vector<uint16_t>& a, size_t m) {
    if (L <= 128) return offsets_coded<128>(a, m);
    if (L <= 256) return offsets_coded<256>(a, m);
    if (L <= 384) return offsets_coded<384>(a, m);
    return offsets_coded<512>(a, m);
}

std::string lzma2_of(const std::string& dir, const std::string& name, const void* data, size_t n,
                     int level, int threads) {
    std::string in = dir + "/" + name + ".bin", out = dir + "/" + name + ".lzma2";
    write_file(in, data, n);
    lzma2::lzma2_compress(in.c_str(), out.c_str(), level, threads);
    std::string s = read_file(out);
    unlink(in.c_str());
    unlink(out.c_str());
    return s;
}

void put_u64_blob(std::ostream& o, const std::string& s) {
    uint64_t n = s.size();
    o.write(reinterpret_cast<const char*>(&n), 8);
    o.write(s.data(), s.size());
}

std::string compressed(const void* src, size_t n, uint8_t coder, int param, double est) {
    std::ostringstream o;
    writeCompressed(o, static_cast<const char*>(src), n, coder, 3, param, est);
    return o.str();
}

template <class T>
std::string pe_id_to_pos(const std::vector<uint64_t>& id_to_pos, const std::string& dir, int level, int thr) {
    // util.cuh:345-442
    std::ostringstream out;
    std::vector<T> base, notbase;
    std::vector<uint8_t> offFlag, offFirst, dFlag, dFirst;
    std::vector<uint16_t> offVal;
    std::vector<int16_t> dVal;
    const uint32_t pairs = uint32_t(id_to_pos.size() / 2);
    std::vector<uint32_t> rank;
    for (uint32_t i = 0; i < id_to_pos.size(); i += 2) {
        base.push_back(T(id_to_pos[i]));
        rank.push_back(i >> 1);
    }
    std::stable_sort(rank.begin(), rank.end(), [&](uint32_t a, uint32_t b) { return base[a] < base[b]; });
    int64_t refPrev = 0, prev = 0;
    bool match = false;
    for (uint32_t q = 0; q < pairs; ++q) {
        uint32_t i = rank[q] * 2;
        bool before = id_to_pos[i] < id_to_pos[i + 1];
        T rel = before ? T(id_to_pos[i + 1] - id_to_pos[i]) : T(id_to_pos[i] - id_to_pos[i + 1]);
        bool in16 = rel <= 0xFFFF;
        offFlag.push_back(in16);
        if (in16) {
            offFirst.push_back(before);
            offVal.push_back(uint16_t(rel));
            continue;
        }
        int64_t delta = int64_t(rel) - refPrev;
        bool d16 = delta <= INT16_MAX && delta >= INT16_MIN;
        dFlag.push_back(d16);
        if (d16) {
            match = true;
            dFirst.push_back(before);
            dVal.push_back(int16_t(delta));
            refPrev = int64_t(rel);
        } else {
            if (!match || refPrev != prev) refPrev = int64_t(rel);
            notbase.push_back(T(id_to_pos[i + 1]));
            match = false;
        }
        prev = int64_t(rel);
    }
    put_u64_blob(out, lzma2_of(dir, "base_pair_pos", base.data(), base.size() * sizeof(T), level, thr));
    out << compressed(offFlag.data(), offFlag.size(), PPMD7_CODER, 3, COMPRESSION_ESTIMATION_UINT8_BITMAP);
    out << compressed(offFirst.data(), offFirst.size(), PPMD7_CODER, 3, COMPRESSION_ESTIMATION_UINT8_BITMAP);
    out << compressed(offVal.data(), offVal.size() * 2, PPMD7_CODER, 3, 1);
    out << compressed(dFlag.data(), dFlag.size(), PPMD7_CODER, 3, COMPRESSION_ESTIMATION_UINT8_BITMAP);
    out << compressed(dFirst.data(), dFirst.size(), PPMD7_CODER, 3, COMPRESSION_ESTIMATION_UINT8_BITMAP);
    out << compressed(dVal.data(), dVal.size() * 2, PPMD7_CODER, 3, 1);
    put_u64_blob(out, lzma2_of(dir, "not_base_pair_pos", notbase.data(), notbase.size() * sizeof(T), level, thr));
    return out.str();
}

std::string pe_order_coded(const std::vector<uint32_t>& order, const std::string& dir, int level, int thr) {
    // util.cuh:444-525
    std::ostringstream out;
    std::vector<uint8_t> offPair, nonOffPair, off8Flag, off8Val, d8Flag;
    std::vector<int8_t> d8Val;
    std::vector<uint32_t> offs;
    std::vector<uint8_t> visit(order.size(), 0);
    std::vector<uint32_t> index(order.size());
    for (uint32_t i = 0; i < order.size(); ++i) index[order[i]] = i;
    int64_t refPrev = 0, prev = 0;
    bool match = false;
    for (uint32_t oi = 0; oi < order.size(); ++oi) {
        if (visit[oi]) continue;
        uint32_t o = order[oi];
        uint32_t po = o % 2 ? o - 1 : o + 1;
        uint32_t pi = index[po];
        visit[pi] = 1;
        int64_t d = int64_t(pi) - int64_t(oi);
        off8Flag.push_back(d <= 255);
        if (d <= 255) {
            off8Val.push_back(uint8_t(d));
            offPair.push_back(o % 2);
            continue;
        }
        nonOffPair.push_back(o % 2);
        int64_t delta = d - refPrev;
        bool d8 = delta >= INT8_MIN && delta <= INT8_MAX;
        d8Flag.push_back(d8);
        if (d8) {
            match = true;
            d8Val.push_back(int8_t(delta));
            refPrev = d;
        } else {
            if (!match || refPrev != prev) refPrev = d;
            offs.push_back(uint32_t(d));
            match = false;
        }
        prev = d;
    }
    out << compressed(off8Flag.data(), off8Flag.size(), PPMD7_CODER, 3, COMPRESSION_ESTIMATION_UINT8_BITMAP);
    out << compressed(off8Val.data(), off8Val.size(), PPMD7_CODER, 2, 1);
    out << compressed(d8Flag.data(), d8Flag.size(), PPMD7_CODER, 3, COMPRESSION_ESTIMATION_UINT8_BITMAP);
    out << compressed(offPair.data(), offPair.size(), PPMD7_CODER, 2, COMPRESSION_ESTIMATION_UINT8_BITMAP);
    out << compressed(nonOffPair.data(), nonOffPair.size(), PPMD7_CODER, 2, COMPRESSION_ESTIMATION_UINT8_BITMAP);
    put_u64_blob(out, lzma2_of(dir, "delta", d8Val.data(), d8Val.size(), level, thr));
    put_u64_blob(out, lzma2_of(dir, "offset", offs.data(), offs.size() * 4, level, thr));
    return out.str();
}

}  // namespace

// Block body in the reference layout (compress.cu:1364-1366, 1911-1921,
// 2017-2146; read back by decompress.cu:760-814).
std::string encode_block(const Params& p, const BlockStreams& s, const std::string& dir, const std::string& bsc) {
    std::ostringstream o;
    o.write(reinterpret_cast<const char*>(&s.reads_count), 4);
    o.write(s.decoder_table, 16);
    const uint64_t joined = s.ref_size + s.unmap_ref_size + s.unmap_n_ref_size;
    const uint8_t join_std = joined <= 0xFFFFFFFFull;
    if (p.preserve_order) o.write(reinterpret_cast<const char*>(&join_std), 1);
    const uint8_t ref_std = s.ref_size <= 0xFFFFFFFFull;
    o.write(reinterpret_cast<const char*>(&ref_std), 1);
    const uint64_t sz[3] = {s.ref.size(), s.unmap_ref.size(), s.unmap_n_ref.size()};
    o.write(reinterpret_cast<const char*>(sz), 24);

    if (p.preserve_order) {
        std::string id_pos;
        if (!p.paired_end) {
            if (join_std) {
                std::vector<uint32_t> v(s.id_to_pos.begin(), s.id_to_pos.end());
                id_pos = lzma2_of(dir, "id_pos", v.data(), v.size() * 4, p.flzma2_level, p.flzma2_threads);
            } else {
                id_pos = lzma2_of(dir, "id_pos", s.id_to_pos.data(), s.id_to_pos.size() * 8, p.flzma2_level,
                                  p.flzma2_threads);
            }
        } else {
            id_pos = join_std ? pe_id_to_pos<uint32_t>(s.id_to_pos, dir, p.flzma2_level, p.flzma2_threads)
                              : pe_id_to_pos<uint64_t>(s.id_to_pos, dir, p.flzma2_level, p.flzma2_threads);
        }
        put_u64_blob(o, id_pos);
    }
    {
        std::string in = dir + "/strand_id.txt", out = dir + "/strand_id.bsc";
        write_file(in, s.strand.data(), s.strand.size());
        std::string cmd = bsc + " e " + in + " " + out + " -pm0 -e2 > /dev/null";
        if (std::system(cmd.c_str()) != 0) throw std::runtime_error("bsc failed");
        put_u64_blob(o, read_file(out));
        unlink(in.c_str());
        unlink(out.c_str());
    }
    {
        std::string joined_ref = s.ref + s.unmap_ref + s.unmap_n_ref;
        size_t clen = 0;
        char* v = Compress(clen, joined_ref.data(), joined_ref.size(), VARLEN_DNA_CODER, 3,
                           PgSAHelpers::VarLenDNACoder::getCoderParam(PgSAHelpers::VarLenDNACoder::STATIC_CODES_CODER_PARAM,
                                                                      PgSAHelpers::VarLenDNACoder::AG_EXTENDED_CODES_ID),
                           1);
        put_u64_blob(o, lzma2_of(dir, "ref_var_len_encode", v, clen, p.flzma2_level, p.flzma2_threads));
        delete[] v;
    }
    if (!p.preserve_order) {
        put_u64_blob(o, compressed(s.read_off.data(), s.read_off.size() * 2, PPMD7_CODER, 3, 1));
        put_u64_blob(o, compressed(s.unmap_n_read_off.data(), s.unmap_n_read_off.size() * 2, PPMD7_CODER, 3, 1));
        put_u64_blob(o, compressed(s.unmap_read_off.data(), s.unmap_read_off.size() * 2, PPMD7_CODER, 3, 1));
        if (p.paired_end) put_u64_blob(o, pe_order_coded(s.pe_order, dir, p.flzma2_level, p.flzma2_threads));
    }
    {
        const double est = simpleUintCompressionEstimate(s.ref.size(), ref_std ? 0xFFFFFFFFull : ~0ull);
        const int period = ref_std ? 2 : 3;
        auto map_pair = [&](const std::string& off, const std::string& len) {
            put_u64_blob(o, compressed(off.data(), off.size(), LZMA_CODER, period, est));
            put_u64_blob(o, compressed(len.data(), len.size(), LZMA_CODER, 0, 1));
        };
        map_pair(s.ref_off, s.ref_len_map);
        map_pair(s.unmap_ref_off, s.unmap_ref_len);
        map_pair(s.unmap_n_ref_off, s.unmap_n_ref_len);
    }
    put_u64_blob(o, compressed(s.mis_cnt.data(), s.mis_cnt.size(), PPMD7_CODER, 2, 1));
    put_u64_blob(o, compressed(s.mis_base.data(), s.mis_base.size(), PPMD7_CODER, 2, COMPRESSION_ESTIMATION_MIS_SYM));
    const uint8_t mm = uint8_t(p.max_mismatch);
    o.write(reinterpret_cast<const char*>(&mm), 1);
    for (int m = 1; m <= p.max_mismatch; ++m) put_u64_blob(o, offsets_for(p.read_len, s.mis_off[m], m));
    return o.str();
}

std::string read_file_pub(const std::string& path) { return read_file(path); }
void write_file_pub(const std::string& path, const void* data, size_t n) { write_file(path, data, n); }

// ---------------------------------------------------------------- ingest

struct RawBlock {
    std::vector<char> seqs;  // reads_count x L, block id order
    size_t count = 0;
};

// preprocess.cpp:66-254 block split: 50 MB windows (25 MB per file for
// paired end) cut at a record boundary; a block closes once the bytes read
// since the last cut exceed block_ratio of the input.
std::vector<RawBlock> split_fastq(const std::string& f1, const std::string& f2, int& L, double ratio) {
    std::string a = read_file(f1), b;
    const bool pe = !f2.empty();
    if (pe) {
        b = read_file(f2);
        if (a.size() != b.size()) throw std::runtime_error("paired-end file size isn't equal");
    }
    {
        size_t e1 = a.find('\n'), e2 = a.find('\n', e1 + 1);
        L = int(e2 - e1 - 1);
    }
    const size_t fq = a.size();
    const size_t block_bytes = pe ? size_t(2 * double(fq) * ratio) : size_t(double(fq) * ratio);
    const size_t win = pe ? 25000000 : 50000000;
    std::vector<RawBlock> blocks(1);
    size_t total = 0, last_total = 0;
    while (total < fq) {
        const char* buf = a.data() + total;
        const char* buf2 = pe ? b.data() + total : nullptr;
        size_t end = std::min(win, fq - total);
        total += end;
        if (total < fq) {
            long fl = 0;
            if (buf[0] != '@') throw std::runtime_error("io_buffer doesn't start with @");
            while (buf[fl] != '\n') fl++;
            size_t ne = end - fl;
            int eq = 0;
            while (ne > 0) {
                if (buf[ne - 1] == '\n' && buf[ne] == '@') {
                    for (long j = 0; j < fl; ++j) {
                        if (buf[j] == buf[ne + j]) {
                            if (++eq > 5) goto cut;
                        } else {
                            eq = 0;
                        }
                    }
                }
                ne--;
            }
            // no boundary: the reference re-reads the same window forever
            throw std::runtime_error("no record boundary found in a 50 MB window");
        cut:
            total -= (end - ne);
            end = ne;
        }
        size_t i = 0, j = 0;
        auto take = [&](const char* s, size_t& k) {
            while (s[k++] != '\n') {}
            size_t st = k;
            while (s[k] != '\n') k++;
            if (long(k - st) != L) throw std::runtime_error("read length isn't fix");
            RawBlock& rb = blocks.back();
            rb.seqs.insert(rb.seqs.end(), s + st, s + k);
            rb.count++;
            k++;
            while (s[k++] != '\n') {}
            while (s[k++] != '\n') {}
        };
        while (i < end) {
            take(buf, i);
            if (pe) take(buf2, j);
        }
        size_t brb = total - last_total;
        if (pe) brb *= 2;
        if (brb > block_bytes) {
            blocks.emplace_back();
            last_total = total;
        }
    }
    if (blocks.back().count == 0) blocks.pop_back();
    if (blocks.size() >= 255) throw std::runtime_error("too many blocks");
    return blocks;
}

BlockInput make_block_input(const Params& p, const RawBlock& rb, std::vector<uint64_t>& db) {
    BlockInput in;
    const int L = p.read_len;
    db.assign(rb.count * p.unit, 0);
    std::vector<uint8_t> hn(rb.count);
    pack_reads(rb.seqs.data(), rb.count, L, db.data(), hn.data());
    in.db = db.data();
    in.reads_count = rb.count;
    for (size_t i = 0; i < rb.count; ++i) {
        if (hn[i]) {
            in.n_ids.push_back(uint32_t(i));
            in.nreads.insert(in.nreads.end(), rb.seqs.data() + i * L, rb.seqs.data() + (i + 1) * L);
        } else {
            in.reads_id.push_back(uint32_t(i));
        }
    }
    return in;
}

}  // namespace oracle

// ---------------------------------------------------------------- C API

namespace {
struct Handle {
    oracle::Params p;
    std::vector<uint64_t> db;
    std::vector<uint8_t> has_n;
    oracle::BlockStreams s;
    std::vector<uint8_t> hq_rec;  // packed Record view: u32 id, u8 n, u8 strand, u16 0, u64 pos
    std::vector<uint8_t> all_rec;
    std::map<std::string, std::string> extra;
};

template <class V>
void view(const V& v, const void** ptr, uint64_t* bytes) {
    *ptr = v.data();
    *bytes = v.size() * sizeof(typename V::value_type);
}
}  // namespace

extern "C" {

// Runs the oracle on one block.  `seqs` holds n reads of length L (ASCII),
// in block id order (paired end: mates interleaved).  `picks` (npicks pairs
// of overlap pass and suffix read id, may be null) replays another
// serialisation of the contested overlap runs: in that pass the suffix is
// visited before the others.
void* oracle_block_new_picks(const char* seqs, uint64_t n, int L, int po, int pe, int threads, const uint32_t* picks,
                             uint64_t npicks) {
    auto* h = new Handle;
    h->p = oracle::Params::derive(L, po != 0, pe != 0);
    oracle::RawBlock rb;
    rb.seqs.assign(seqs, seqs + n * L);
    rb.count = n;
    oracle::BlockInput in = oracle::make_block_input(h->p, rb, h->db);
    for (uint64_t i = 0; i < npicks; ++i) in.contest_picks.push_back({int(picks[2 * i]), picks[2 * i + 1]});
    h->has_n.assign(n, 0);
    for (uint32_t id : in.n_ids) h->has_n[id] = 1;
    oracle::compress_block(h->p, in, h->s, threads);
    auto flat = [](const std::vector<oracle::Record>& rs, std::vector<uint8_t>& outv) {
        for (const auto& r : rs) {
            uint8_t b[16] = {0};
            std::memcpy(b, &r.read_id, 4);
            b[4] = r.is_n;
            b[5] = r.strand;
            std::memcpy(b + 8, &r.pos, 8);
            outv.insert(outv.end(), b, b + 16);
        }
    };
    flat(h->s.hq.records, h->hq_rec);
    flat(h->s.records, h->all_rec);
    return h;
}

void* oracle_block_new(const char* seqs, uint64_t n, int L, int po, int pe, int threads) {
    return oracle_block_new_picks(seqs, n, L, po, pe, threads, nullptr, 0);
}

int oracle_block_get(void* hv, const char* name, const void** ptr, uint64_t* bytes) {
    auto* h = static_cast<Handle*>(hv);
    const auto& s = h->s;
    std::string n(name);
    if (n == "packed") view(h->db, ptr, bytes);
    else if (n == "has_n") view(h->has_n, ptr, bytes);
    else if (n == "sorted_ids") view(s.sorted_ids, ptr, bytes);
    else if (n == "next") view(s.next, ptr, bytes);
    else if (n == "prev") view(s.prev, ptr, bytes);
    else if (n == "offset") view(s.offset, ptr, bytes);
    else if (n == "ref_ids") view(s.ref_ids, ptr, bytes);
    else if (n == "unmatch_ids") view(s.unmatch_ids, ptr, bytes);
    else if (n == "hq_seq") view(s.hq.seq, ptr, bytes);
    else if (n == "hq_records") view(h->hq_rec, ptr, bytes);
    else if (n == "records") view(h->all_rec, ptr, bytes);
    else if (n == "map_mm") view(s.map.mm, ptr, bytes);
    else if (n == "map_strand") view(s.map.strand, ptr, bytes);
    else if (n == "map_pos") view(s.map.pos, ptr, bytes);
    else if (n == "contests") view(s.contests, ptr, bytes);  // u32 (pass, run, suffix, prefix) per member
    else if (n == "ref") view(s.ref, ptr, bytes);
    else if (n == "unmap_ref") view(s.unmap_ref, ptr, bytes);
    else if (n == "unmap_n_ref") view(s.unmap_n_ref, ptr, bytes);
    else if (n == "strand") view(s.strand, ptr, bytes);
    else if (n == "mis_cnt") view(s.mis_cnt, ptr, bytes);
    else if (n == "mis_base") view(s.mis_base, ptr, bytes);
    else if (n == "read_off") view(s.read_off, ptr, bytes);
    else if (n == "unmap_read_off") view(s.unmap_read_off, ptr, bytes);
    else if (n == "unmap_n_read_off") view(s.unmap_n_read_off, ptr, bytes);
    else if (n == "pe_order") view(s.pe_order, ptr, bytes);
    else if (n == "id_to_pos") view(s.id_to_pos, ptr, bytes);
    else if (n == "ref_off") view(s.ref_off, ptr, bytes);
    else if (n == "ref_len_map") view(s.ref_len_map, ptr, bytes);
    else if (n == "unmap_ref_off") view(s.unmap_ref_off, ptr, bytes);
    else if (n == "unmap_ref_len") view(s.unmap_ref_len, ptr, bytes);
    else if (n == "unmap_n_ref_off") view(s.unmap_n_ref_off, ptr, bytes);
    else if (n == "unmap_n_ref_len") view(s.unmap_n_ref_len, ptr, bytes);
    else if (n == "decoder_table") { *ptr = s.decoder_table; *bytes = 16; }
    else if (n.rfind("mis_off_", 0) == 0) {
        int m = std::atoi(n.c_str() + 8);
        if (m < 1 || m > h->p.max_mismatch) return -1;
        view(s.mis_off[m], ptr, bytes);
    } else if (n == "sizes") {
        std::string& e = h->extra["sizes"];
        uint64_t v[6] = {s.ref_size, s.unmap_ref_size, s.unmap_n_ref_size, s.ref.size(), s.unmap_ref.size(),
                         s.unmap_n_ref.size()};
        e.assign(reinterpret_cast<const char*>(v), sizeof(v));
        view(e, ptr, bytes);
    } else {
        return -1;
    }
    return 0;
}

// Codes the block into the reference block layout; returns its size and a
// malloc'd buffer in *out (free with oracle_buf_free).
uint64_t oracle_block_encode(void* hv, const char* tmpdir, const char* bsc, char** out) {
    auto* h = static_cast<Handle*>(hv);
    std::string b = oracle::encode_block(h->p, h->s, tmpdir, bsc);
    *out = static_cast<char*>(std::malloc(b.size() ? b.size() : 1));
    std::memcpy(*out, b.data(), b.size());
    return b.size();
}

void oracle_buf_free(char* p) { std::free(p); }
void oracle_block_free(void* hv) { delete static_cast<Handle*>(hv); }

// Whole-file compressor with the reference's CLI semantics; writes
// <working_dir>/<name>.curc.  Returns 0 on success.
int oracle_compress_files(const char* f1, const char* f2, const char* working_dir, const char* name, double ratio,
                          int po, const char* bsc, int threads) {
    try {
        int L = 0;
        std::string s2 = f2 ? f2 : "";
        auto blocks = oracle::split_fastq(f1, s2, L, ratio);
        oracle::Params p = oracle::Params::derive(L, po != 0, !s2.empty());
        if (p.unit > 16) throw std::runtime_error("Read length must be less than 512");
        std::string tmp = std::string(working_dir) + "/oracle_tmp_XXXXXX";
        if (!mkdtemp(&tmp[0])) throw std::runtime_error("mkdtemp failed");
        std::ofstream out(std::string(working_dir) + "/" + name + ".curc", std::ios::binary);
        uint8_t hdr[5] = {uint8_t(po != 0), uint8_t(!s2.empty()), uint8_t(L & 0xFF), uint8_t(L >> 8),
                          uint8_t(blocks.size())};
        out.write(reinterpret_cast<const char*>(hdr), 5);
        for (auto& rb : blocks) {
            std::vector<uint64_t> db;
            oracle::BlockInput in = oracle::make_block_input(p, rb, db);
            oracle::BlockStreams s;
            oracle::compress_block(p, in, s, threads);
            std::string body = oracle::encode_block(p, s, tmp, bsc);
            out.write(body.data(), body.size());
        }
        rmdir(tmp.c_str());
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "oracle: %s\n", e.what());
        return 1;
    }
}
}

namespace lzma2 {
void lzma2_decompress(const char* infile, const char* outfile);
}

extern "C" {

// Decodes one writeCompressed payload (LzmaLib.cpp:539-552 container).
uint64_t oracle_read_compressed(const char* buf, uint64_t n, char** out) {
    std::istringstream in(std::string(buf, n));
    std::string dest;
    readCompressed(in, dest);
    *out = static_cast<char*>(std::malloc(dest.size() ? dest.size() : 1));
    std::memcpy(*out, dest.data(), dest.size());
    return dest.size();
}

// Decodes the ref.lzma2 payload: fast-lzma2, then the VarLenDNA coder, into
// the joined pseudogenome of `total` symbols.
uint64_t oracle_decode_ref(const char* buf, uint64_t n, uint64_t total, const char* tmpdir, char** out) {
    std::string in = std::string(tmpdir) + "/ref_in.lzma2", mid = std::string(tmpdir) + "/ref_mid.bin";
    oracle::write_file_pub(in, buf, n);
    lzma2::lzma2_decompress(in.c_str(), mid.c_str());
    std::string enc = oracle::read_file_pub(mid);
    unlink(in.c_str());
    unlink(mid.c_str());
    *out = static_cast<char*>(std::malloc(total ? total : 1));
    Uncompress(*out, total, enc.data(), enc.size(), VARLEN_DNA_CODER);
    return total;
}

// Decodes a mismatch-offset stream of mismatch count m (util.cuh:307-343)
// holding `records` records; writes uint16 values.
uint64_t oracle_decode_offsets(const char* buf, uint64_t n, int read_len, int m, uint64_t records, uint16_t* out) {
    std::vector<char> copy(buf, buf + n);
    copy.resize(n + 64, 0);
    auto run = [&](auto tag) {
        constexpr size_t MaxL = decltype(tag)::value;
        RangeCoder rc{};
        rc.input(copy.data());
        rc.StartDecode();
        SIMPLE_MODEL<2> flag;
        SIMPLE_MODEL<MaxL / 2 + 1> first;
        SIMPLE_MODEL<MaxL> value;
        uint64_t k = 0;
        for (uint64_t r = 0; r < records; ++r) {
            out[k++] = flag.decodeSymbol(&rc);
            out[k++] = first.decodeSymbol(&rc);
            if (m > 1) {
                out[k++] = value.decodeSymbol(&rc);
                if (m > 2)
                    for (int t = 1; t < m; ++t) out[k++] = value.decodeSymbol(&rc);
            }
        }
        rc.FinishDecode();
        return k;
    };
    if (read_len <= 128) return run(std::integral_constant<size_t, 128>{});
    if (read_len <= 256) return run(std::integral_constant<size_t, 256>{});
    if (read_len <= 384) return run(std::integral_constant<size_t, 384>{});
    return run(std::integral_constant<size_t, 512>{});
}
}

extern "C" {

// The block split of split_fastq (preprocess.cpp:66-254): block count,
// read length, reads per block (counts, up to 255 entries) and all blocks'
// reads concatenated (*seqs, freed with oracle_buf_free).  Returns 0, or -1
// with the message in *seqs.
int oracle_split_fastq(const char* f1, const char* f2, double ratio, uint32_t* nblocks, int* read_len,
                       uint64_t* counts, char** seqs, uint64_t* seq_bytes) {
    try {
        int L = 0;
        auto blocks = oracle::split_fastq(f1, f2 ? f2 : "", L, ratio);
        size_t total = 0;
        for (const auto& b : blocks) total += b.seqs.size();
        char* out = static_cast<char*>(std::malloc(total ? total : 1));
        size_t off = 0;
        for (size_t i = 0; i < blocks.size(); ++i) {
            counts[i] = blocks[i].count;
            if (!blocks[i].seqs.empty()) std::memcpy(out + off, blocks[i].seqs.data(), blocks[i].seqs.size());
            off += blocks[i].seqs.size();
        }
        *nblocks = uint32_t(blocks.size());
        *read_len = L;
        *seqs = out;
        *seq_bytes = total;
        return 0;
    } catch (const std::exception& e) {
        const std::string m = e.what();
        char* out = static_cast<char*>(std::malloc(m.size() + 1));
        std::memcpy(out, m.c_str(), m.size() + 1);
        *seqs = out;
        return -1;
    }
}
}
