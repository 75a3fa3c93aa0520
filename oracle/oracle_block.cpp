// CPU oracle for the CURC pseudogenome path -- TEST INFRASTRUCTURE ONLY.
// Block driver and stream emission: compress.cu:1349-2148 without the coders.
#include <algorithm>
#include <cstring>
#include <numeric>
#include <stdexcept>

#include "oracle.hpp"

namespace oracle {

namespace {

// Mismatch-offset coding of one record (compress.cu:1847-1886): direction
// flag, first offset from the chosen end, then either the gap (2 mismatches)
// or min_gap-1 followed by each gap minus min_gap.
void encode_offsets(const std::vector<uint16_t>& mo, int L, std::vector<uint16_t>& out) {
    const size_t m = mo.size();
    if (mo[0] < (L - 1 - mo[m - 1])) {
        out.push_back(0);
        out.push_back(mo[0]);
        if (m > 1) {
            if (m == 2) {
                out.push_back(uint16_t(mo[1] - mo[0] - 1));
            } else {
                uint32_t mn = 0xFFFFFFFFu;
                for (size_t i = 1; i < m; ++i) mn = std::min<uint32_t>(mn, mo[i] - mo[i - 1]);
                out.push_back(uint16_t(mn - 1));
                for (size_t i = 1; i < m; ++i) out.push_back(uint16_t(mo[i] - mo[i - 1] - mn));
            }
        }
    } else {
        out.push_back(1);
        out.push_back(uint16_t(L - 1 - mo[m - 1]));
        if (m > 1) {
            if (m == 2) {
                out.push_back(uint16_t(mo[1] - mo[0] - 1));
            } else {
                uint32_t mn = 0xFFFFFFFFu;
                for (size_t i = m - 1; i > 0; --i) mn = std::min<uint32_t>(mn, mo[i] - mo[i - 1]);
                out.push_back(uint16_t(mn - 1));
                for (size_t i = m - 1; i > 0; --i) out.push_back(uint16_t(mo[i] - mo[i - 1] - mn));
            }
        }
    }
}

}  // namespace

void compress_block(const Params& p, const BlockInput& in, BlockStreams& out, int threads) {
    const int L = p.read_len, W = p.unit;
    const size_t n = in.reads_count;
    out.reads_count = uint32_t(n);

    // a2 (compress.cu:1389-1420)
    out.next.assign(n, INVALID);
    out.prev.assign(n, INVALID);
    out.offset.assign(n, INVALOFF);
    out.sorted_ids = in.reads_id;
    sort_dedupe(in.db, W, out.sorted_ids, out.next.data(), out.prev.data(), out.offset.data());
    // a3 + a4
    OverlapControl ctl;
    ctl.picks = in.contest_picks;
    ctl.log = &out.contests;
    overlap_link(p, in.db, out.sorted_ids, out.next.data(), out.prev.data(), out.offset.data(), &ctl, threads);
    // a5
    chain_filter(n, out.sorted_ids, out.next.data(), out.prev.data(), out.offset.data(), out.ref_ids,
                 out.unmatch_ids);
    // a6 (compress.cu:1576-1591)
    {
        std::vector<uint32_t> pre, suf;
        for (uint32_t id : out.ref_ids) {
            if (out.prev[id] == INVALID) pre.push_back(id);
            if (out.next[id] == INVALID) suf.push_back(id);
        }
        full_match_packed(p, in.db, pre, suf, out.next.data(), out.prev.data(), out.offset.data());
    }
    // a8 (compress.cu:1612-1620)
    Pseudogenome& hq = out.hq;
    assemble_packed(in.db, L, W, out.ref_ids, out.next.data(), out.prev.data(), out.offset.data(), n, hq);
    std::vector<uint64_t> hq_bin = pack_ref(hq.seq);

    // a9 (compress.cu:1622-1640)
    const size_t U = out.unmatch_ids.size(), NN = in.n_ids.size();
    std::vector<uint64_t> udb(U * W);
    for (size_t i = 0; i < U; ++i)
        std::memcpy(&udb[i * W], in.db + size_t(out.unmatch_ids[i]) * W, W * sizeof(uint64_t));
    map_reads(p, hq_bin.data(), hq.seq.size(), udb.data(), U, in.nreads.data(), NN, out.map, threads);
    const MapResult& mr = out.map;
    std::vector<uint32_t> unmap_local;  // indices into unmatch_ids
    std::vector<uint32_t> unmap_n;      // N-local indices
    std::vector<Record> map_rec;
    std::vector<uint8_t> map_mm;
    for (size_t i = 0; i < U + NN; ++i) {
        if (mr.mm[i] <= p.max_mismatch) {
            uint32_t rid = i < U ? out.unmatch_ids[i] : uint32_t(i - U);
            map_rec.push_back({rid, uint8_t(i >= U), mr.strand[i], mr.pos[i]});
            map_mm.push_back(mr.mm[i]);
        } else if (i < U) {
            unmap_local.push_back(uint32_t(i));
        } else {
            unmap_n.push_back(uint32_t(i - U));
        }
    }

    // a11 non-N (compress.cu:1649-1722): reads renumbered 0..n-1 in list
    // order, which is lexicographic, then full match + assembly
    Pseudogenome lq;
    if (!unmap_local.empty()) {
        const size_t m = unmap_local.size();
        std::vector<uint64_t> ldb(m * W);
        for (size_t i = 0; i < m; ++i)
            std::memcpy(&ldb[i * W], &udb[size_t(unmap_local[i]) * W], W * sizeof(uint64_t));
        std::vector<uint32_t> nx(m, INVALID), pv(m, INVALID);
        std::vector<uint16_t> of(m, INVALOFF);
        std::vector<uint32_t> seq(m);
        std::iota(seq.begin(), seq.end(), 0);
        full_match_packed(p, ldb.data(), seq, seq, nx.data(), pv.data(), of.data());
        assemble_packed(ldb.data(), L, W, seq, nx.data(), pv.data(), of.data(), m, lq);
        for (auto& r : lq.records) r.read_id = out.unmatch_ids[unmap_local[r.read_id]];
    }
    // a7 + a11 N (compress.cu:1724-1728)
    Pseudogenome lqn;
    if (!unmap_n.empty()) {
        std::vector<uint32_t> nx, pv;
        std::vector<uint16_t> of;
        full_match_ascii(p, in.nreads.data(), unmap_n, NN, nx, pv, of);
        std::vector<uint32_t> sorted = unmap_n;
        std::stable_sort(sorted.begin(), sorted.end(), [&](uint32_t a, uint32_t b) {
            return std::memcmp(&in.nreads[size_t(a) * L], &in.nreads[size_t(b) * L], L) < 0;
        });
        assemble_ascii(in.nreads.data(), L, sorted, nx.data(), pv.data(), of.data(), NN, lqn);
    }

    // a10 (compress.cu:1730-1961)
    std::vector<Record> rec = hq.records;
    std::vector<uint8_t> mis(rec.size(), 0);
    rec.insert(rec.end(), map_rec.begin(), map_rec.end());
    mis.insert(mis.end(), map_mm.begin(), map_mm.end());
    auto orig = [&](const Record& r) { return r.is_n ? in.n_ids[r.read_id] : r.read_id; };
    {
        std::vector<uint32_t> ord(rec.size());
        std::iota(ord.begin(), ord.end(), 0);
        if (!p.preserve_order)
            std::stable_sort(ord.begin(), ord.end(), [&](uint32_t a, uint32_t b) { return rec[a].pos < rec[b].pos; });
        else
            std::stable_sort(ord.begin(), ord.end(), [&](uint32_t a, uint32_t b) { return orig(rec[a]) < orig(rec[b]); });
        std::vector<Record> r2(rec.size());
        std::vector<uint8_t> m2(rec.size());
        for (size_t i = 0; i < ord.size(); ++i) { r2[i] = rec[ord[i]]; m2[i] = mis[ord[i]]; }
        rec.swap(r2);
        mis.swap(m2);
    }
    if (p.preserve_order) out.id_to_pos.assign(n, 0);
    out.strand.resize(rec.size());
    out.mis_off.assign(p.max_mismatch + 1, {});
    std::string ctx_stream, base_stream;
    if (!p.preserve_order) out.read_off.resize(rec.size());
    for (size_t i = 0; i < rec.size(); ++i) {
        const Record& r = rec[i];
        if (p.preserve_order) {
            out.id_to_pos[orig(r)] = r.pos;
        } else {
            if (p.paired_end) out.pe_order.push_back(orig(r));
            out.read_off[i] = i == 0 ? 0 : uint16_t(r.pos - rec[i - 1].pos);
        }
        out.strand[i] = char('0' + r.strand);
        if (mis[i] == 0) continue;
        std::vector<uint16_t> mo;
        for (int q = 0; q < L; ++q) {
            char rb;
            int src = r.strand == 0 ? q : L - 1 - q;
            if (!r.is_n)
                rb = base_at(in.db + size_t(r.read_id) * W, src);
            else
                rb = in.nreads[size_t(r.read_id) * L + src];
            if (r.strand == 1) rb = comp_base(rb);
            char gb = hq.seq[r.pos + q];
            if (gb != rb) {
                ctx_stream.push_back(gb);
                base_stream.push_back(rb);
                mo.push_back(uint16_t(q));
            }
        }
        if (mo.size() != mis[i]) throw std::runtime_error("oracle: mismatch count disagrees with mapping");
        encode_offsets(mo, L, out.mis_off[mis[i]]);
    }
    out.mis_cnt = mis;
    out.records = rec;
    // context recode (compress.cu:1889-1929): per context, destination bases
    // ranked by descending frequency, ties in listed order (insertion sort)
    {
        static size_t freq[256][256];
        std::memset(freq, 0, sizeof(freq));
        for (size_t i = 0; i < base_stream.size(); ++i) freq[uint8_t(ctx_stream[i])][uint8_t(base_stream[i])]++;
        struct Ctx { char c; char d[4]; };
        const Ctx ctxs[4] = {{'A', {'C', 'G', 'N', 'T'}}, {'T', {'A', 'C', 'G', 'N'}},
                             {'C', {'A', 'G', 'N', 'T'}}, {'G', {'A', 'C', 'N', 'T'}}};
        for (int t = 0; t < 4; ++t) {
            const Ctx& c = ctxs[t];
            int idx[4] = {0, 1, 2, 3};
            std::stable_sort(idx, idx + 4, [&](int a, int b) {
                return freq[uint8_t(c.c)][uint8_t(c.d[a])] > freq[uint8_t(c.c)][uint8_t(c.d[b])];
            });
            for (int i = 0; i < 4; ++i) freq[uint8_t(c.c)][uint8_t(c.d[idx[i]])] = size_t(i);
            for (char ch : c.d) out.decoder_table[t * 4 + freq[uint8_t(c.c)][uint8_t(ch)]] = ch;
        }
        out.mis_base.resize(base_stream.size());
        for (size_t i = 0; i < base_stream.size(); ++i)
            out.mis_base[i] = char(freq[uint8_t(ctx_stream[i])][uint8_t(base_stream[i])]);
    }

    // unmapped reference offsets / order (compress.cu:1968-2006)
    if (!p.preserve_order) {
        uint64_t last = 0;
        for (const Record& r : lq.records) {
            if (p.paired_end) out.pe_order.push_back(r.read_id);
            out.unmap_read_off.push_back(uint16_t(L - (r.pos - last)));
            last = r.pos;
        }
        last = 0;
        for (const Record& r : lqn.records) {
            if (p.paired_end) out.pe_order.push_back(in.n_ids[r.read_id]);
            out.unmap_n_read_off.push_back(uint16_t(L - (r.pos - last)));
            last = r.pos;
        }
    } else {
        for (const Record& r : lq.records) out.id_to_pos[r.read_id] = hq.seq.size() + r.pos;
        for (const Record& r : lqn.records)
            out.id_to_pos[in.n_ids[r.read_id]] = hq.seq.size() + lq.seq.size() + r.pos;
    }
    out.ref_size = hq.seq.size();
    out.unmap_ref_size = lq.seq.size();
    out.unmap_n_ref_size = lqn.seq.size();

    // a12 (compress.cu:2053-2069)
    out.ref = hq.seq;
    out.unmap_ref = lq.seq;
    out.unmap_n_ref = lqn.seq;
    if (hq.seq.size() >= 36) {
        RefMatcherIndex ix;
        refmatch_index(hq_bin.data(), hq.seq.size(), ix);
        if (!out.unmap_ref.empty())
            refmatch_apply(ix, out.unmap_ref, false, false, out.unmap_ref_off, out.unmap_ref_len, threads);
        if (!out.unmap_n_ref.empty())
            refmatch_apply(ix, out.unmap_n_ref, true, false, out.unmap_n_ref_off, out.unmap_n_ref_len, threads);
        refmatch_apply(ix, out.ref, false, true, out.ref_off, out.ref_len_map, threads);
    }
}

}  // namespace oracle
