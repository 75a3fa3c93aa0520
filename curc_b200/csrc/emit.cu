// a10 + a11: stream emission and the unmapped pseudogenomes.
//
// Reference: compress.cu:1642-1729 (unmapped references), 1730-1961
// (records -> streams), 1964-2006 (unmapped offsets / order).
//
// Records (pseudogenome reads, then mapped reads) are ordered by position
// (or by read id with --preserve_order) with a stable radix sort; each record
// then derives its own mismatches against the pseudogenome in parallel.
// Output slots are fixed beforehand by exclusive scans: mismatch bases by a
// scan of the counts, mismatch offsets per count class by a stable sort of
// the records on their count.
#include <cstring>

#include "block.cuh"

namespace curc {

namespace {

__global__ void map_records_kernel(const uint8_t* __restrict__ mm, const uint8_t* __restrict__ strand,
                                   const uint64_t* __restrict__ pos, uint32_t U, uint32_t NN, int max_mm,
                                   const uint32_t* __restrict__ unmatch_ids, uint8_t* __restrict__ mapped,
                                   uint8_t* __restrict__ unmapped_u, uint8_t* __restrict__ unmapped_n,
                                   DevRecord* __restrict__ rec) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= U + NN) return;
    const bool ok = mm[i] <= max_mm;
    mapped[i] = ok;
    if (i < U) unmapped_u[i] = !ok;
    else unmapped_n[i - U] = !ok;
    DevRecord d;
    d.read_id = i < U ? unmatch_ids[i] : i - U;
    d.is_n = i >= U;
    d.strand = strand[i];
    d.pad = 0;
    d.pos = pos[i];
    rec[i] = d;
}

__global__ void sort_keys_kernel(const DevRecord* __restrict__ rec, uint32_t T, bool po,
                                 const uint32_t* __restrict__ n_ids, uint64_t* __restrict__ key,
                                 uint32_t* __restrict__ idx) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= T) return;
    const DevRecord r = rec[i];
    key[i] = po ? uint64_t(r.is_n ? n_ids[r.read_id] : r.read_id) : r.pos;
    idx[i] = i;
}

__global__ void gather_records_kernel(const DevRecord* __restrict__ rec, const uint8_t* __restrict__ mis,
                                      const uint32_t* __restrict__ idx, uint32_t T, DevRecord* __restrict__ out,
                                      uint8_t* __restrict__ mis_out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= T) return;
    out[i] = rec[idx[i]];
    mis_out[i] = mis[idx[i]];
}

// compress.cu:1798-1813: order / position streams and strand characters.
__global__ void record_streams_kernel(const DevRecord* __restrict__ rec, uint32_t T, bool po, bool pe,
                                      const uint32_t* __restrict__ n_ids, char* __restrict__ strand,
                                      uint16_t* __restrict__ read_off, uint32_t* __restrict__ pe_order,
                                      uint64_t* __restrict__ id_to_pos) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= T) return;
    const DevRecord r = rec[i];
    const uint32_t orig = r.is_n ? n_ids[r.read_id] : r.read_id;
    if (po) {
        id_to_pos[orig] = r.pos;
    } else {
        if (pe) pe_order[i] = orig;
        read_off[i] = i == 0 ? 0 : uint16_t(r.pos - rec[i - 1].pos);
    }
    strand[i] = char('0' + r.strand);
}

__host__ __device__ inline uint32_t class_width(uint32_t m) { return m == 1 ? 2 : (m == 2 ? 3 : m + 2); }

// Records per mismatch count (bins 1..nb-1), counted in shared memory by a
// resident grid and added to hist once per block.
__global__ void __launch_bounds__(256) class_hist_kernel(const uint8_t* __restrict__ mis, uint32_t T, int nb,
                                                         uint32_t* __restrict__ hist) {
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < T; i += gridDim.x * blockDim.x)
        if (mis[i]) atomicAdd(&h[mis[i]], 1u);
    __syncthreads();
    if (int(threadIdx.x) < nb && h[threadIdx.x]) atomicAdd(&hist[threadIdx.x], h[threadIdx.x]);
}

__global__ void class_keys_kernel(const uint32_t* __restrict__ sel, uint32_t c, const uint8_t* __restrict__ mis,
                                  uint32_t* __restrict__ key) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < c) key[t] = mis[sel[t]];
}

// class_rank[record] = position of the record among records with the same
// mismatch count (key sorted stably, so ranks follow record order).
__global__ void class_rank_kernel(const uint32_t* __restrict__ key, const uint32_t* __restrict__ rec_of, uint32_t c,
                                  const uint32_t* __restrict__ class_first, uint32_t* __restrict__ class_rank) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < c) class_rank[rec_of[t]] = t - class_first[key[t]];
}

struct EmitCtx {
    const DevRecord* rec;
    const uint8_t* mis;
    const uint32_t* base_idx;    // exclusive scan of mis
    const uint32_t* class_rank;
    const uint64_t* class_base;  // element offset of each class in off_all
    const uint64_t* db;
    const uint8_t* nreads;
    const uint8_t* ref;          // ASCII pseudogenome
    const uint64_t* packed;      // its 2-bit copy (one zero pad word)
    int L, W;
    uint8_t* ctx;
    uint8_t* base;
    uint16_t* off_all;
    uint32_t* err;
};

// compress.cu:1815-1886 for one record.
__global__ void mismatch_kernel(EmitCtx e, uint32_t T) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= T) return;
    const uint32_t m = e.mis[i];
    if (m == 0) return;
    const DevRecord r = e.rec[i];
    const int L = e.L;
    uint16_t mo[104];
    uint32_t found = 0, bi = e.base_idx[i];
    if (!r.is_n) {
        // packed read against the packed pseudogenome, 32 bases per step: the
        // differing 2-bit groups give the mismatch positions in order
        const uint64_t* rd = e.db + uint64_t(r.read_id) * e.W;
        for (int p0 = 0; p0 < L; p0 += 32) {
            const int nb = L - p0 < 32 ? L - p0 : 32;
            const uint64_t gw = word_unaligned(e.packed, r.pos + p0, nb);
            const uint64_t rw = r.strand == 0 ? word_at(rd, p0, nb) : revcomp_kmer(word_at(rd, L - p0 - nb, nb), nb);
            const uint64_t x = gw ^ rw;
            uint64_t y = (x | (x >> 1)) & 0x5555555555555555ull;  // low bit of each differing group
            while (y) {
                const int bit = 63 - __clzll(y);
                y &= ~(1ull << bit);
                const int t = nb - 1 - bit / 2;  // group index from the first base
                if (found < m) {
                    e.ctx[bi + found] = uint8_t("ACGT"[(gw >> (2 * (nb - 1 - t))) & 3u]);
                    e.base[bi + found] = uint8_t("ACGT"[(rw >> (2 * (nb - 1 - t))) & 3u]);
                    if (found < 104) mo[found] = uint16_t(p0 + t);
                }
                ++found;
            }
        }
    } else {
        const uint8_t* nd = e.nreads + uint64_t(r.read_id) * L;
        const uint8_t* g = e.ref + r.pos;
        for (int p = 0; p < L; ++p) {
            const int src = r.strand == 0 ? p : L - 1 - p;
            char rb = char(nd[src]);
            if (r.strand == 1) rb = comp_char(rb);
            const char gb = char(g[p]);
            if (gb != rb) {
                if (found < m) {
                    e.ctx[bi + found] = uint8_t(gb);
                    e.base[bi + found] = uint8_t(rb);
                    if (found < 104) mo[found] = uint16_t(p);
                }
                ++found;
            }
        }
    }
    if (found != m || m > 104) {
        atomicExch(e.err, 1u);
        return;
    }
    uint16_t* out = e.off_all + e.class_base[m] + uint64_t(e.class_rank[i]) * class_width(m);
    uint32_t k = 0;
    if (mo[0] < (L - 1 - mo[m - 1])) {
        out[k++] = 0;
        out[k++] = mo[0];
        if (m > 1) {
            if (m == 2) {
                out[k++] = uint16_t(mo[1] - mo[0] - 1);
            } else {
                uint32_t mn = 0xFFFFFFFFu;
                for (uint32_t t = 1; t < m; ++t) mn = min(mn, uint32_t(mo[t] - mo[t - 1]));
                out[k++] = uint16_t(mn - 1);
                for (uint32_t t = 1; t < m; ++t) out[k++] = uint16_t(mo[t] - mo[t - 1] - mn);
            }
        }
    } else {
        out[k++] = 1;
        out[k++] = uint16_t(L - 1 - mo[m - 1]);
        if (m > 1) {
            if (m == 2) {
                out[k++] = uint16_t(mo[1] - mo[0] - 1);
            } else {
                uint32_t mn = 0xFFFFFFFFu;
                for (uint32_t t = m - 1; t > 0; --t) mn = min(mn, uint32_t(mo[t] - mo[t - 1]));
                out[k++] = uint16_t(mn - 1);
                for (uint32_t t = m - 1; t > 0; --t) out[k++] = uint16_t(mo[t] - mo[t - 1] - mn);
            }
        }
    }
}

__device__ __forceinline__ int ctx_slot(uint8_t c) {
    switch (c) {
        case 'A': return 0;
        case 'T': return 1;
        case 'C': return 2;
        case 'G': return 3;
        default: return -1;
    }
}
__device__ __forceinline__ int sym_slot(uint8_t c) {
    switch (c) {
        case 'A': return 0;
        case 'C': return 1;
        case 'G': return 2;
        case 'N': return 3;
        case 'T': return 4;
        default: return -1;
    }
}

__global__ void ctx_hist_kernel(const uint8_t* __restrict__ ctx, const uint8_t* __restrict__ base, uint64_t nb,
                                unsigned long long* __restrict__ hist, uint32_t* __restrict__ err) {
    __shared__ unsigned long long h[20];
    if (threadIdx.x < 20) h[threadIdx.x] = 0;
    __syncthreads();
    for (uint64_t j = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < nb; j += uint64_t(gridDim.x) * blockDim.x) {
        const int c = ctx_slot(ctx[j]), b = sym_slot(base[j]);
        if (c < 0 || b < 0) {
            atomicExch(err, 2u);
            continue;
        }
        atomicAdd(&h[c * 5 + b], 1ull);
    }
    __syncthreads();
    if (threadIdx.x < 20 && h[threadIdx.x]) atomicAdd(&hist[threadIdx.x], h[threadIdx.x]);
}

// compress.cu:1889-1921: per context (A, T, C, G) its four possible
// substitutes ranked by descending count, ties in listed order; the table
// maps context and substitute to its rank, and each context's 4 bytes list
// the substitutes by rank.
__global__ void ctx_rank_kernel(const unsigned long long* __restrict__ hist, uint8_t* __restrict__ rank,
                                char* __restrict__ table) {
    if (threadIdx.x != 0) return;
    const char dest[4][4] = {{'C', 'G', 'N', 'T'}, {'A', 'C', 'G', 'N'}, {'A', 'G', 'N', 'T'}, {'A', 'C', 'N', 'T'}};
    for (int c = 0; c < 4; ++c) {
        unsigned long long cnt[4];
        int idx[4];
        for (int d = 0; d < 4; ++d) {
            cnt[d] = hist[c * 5 + sym_slot(uint8_t(dest[c][d]))];
            idx[d] = d;
        }
        for (int a = 1; a < 4; ++a) {  // stable insertion sort, descending
            int v = idx[a], b = a - 1;
            while (b >= 0 && cnt[idx[b]] < cnt[v]) {
                idx[b + 1] = idx[b];
                --b;
            }
            idx[b + 1] = v;
        }
        for (int r = 0; r < 4; ++r) {
            rank[c * 5 + sym_slot(uint8_t(dest[c][idx[r]]))] = uint8_t(r);
            table[c * 4 + r] = dest[c][idx[r]];
        }
    }
}

__global__ void recode_kernel(const uint8_t* __restrict__ ctx, uint8_t* __restrict__ base, uint64_t nb,
                              const uint8_t* __restrict__ rank) {
    for (uint64_t j = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < nb; j += uint64_t(gridDim.x) * blockDim.x) {
        const int c = ctx_slot(ctx[j]), b = sym_slot(base[j]);
        if (c >= 0 && b >= 0) base[j] = rank[c * 5 + b];
    }
}

__global__ void unmapped_offsets_kernel(const DevRecord* __restrict__ rec, uint32_t c, int L, bool po, bool pe,
                                        const uint32_t* __restrict__ id_map, uint64_t pos_base,
                                        uint16_t* __restrict__ off, uint32_t* __restrict__ pe_order,
                                        uint64_t* __restrict__ id_to_pos) {
    // compress.cu:1968-2006: records keep local ids; id_map turns them into
    // block read ids
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c) return;
    const DevRecord r = rec[i];
    const uint32_t orig = id_map[r.read_id];
    if (po) {
        id_to_pos[orig] = pos_base + r.pos;
    } else {
        const uint64_t last = i == 0 ? 0 : rec[i - 1].pos;
        off[i] = uint16_t(L - (r.pos - last));
        if (pe) pe_order[i] = orig;
    }
}

__global__ void widen_u8_kernel(const uint8_t* __restrict__ in, uint32_t* __restrict__ out, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = in[i];
}

__global__ void nonzero_u8_kernel(const uint8_t* __restrict__ in, uint8_t* __restrict__ out, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = in[i] != 0;
}

__global__ void gather_rows_kernel(const uint64_t* __restrict__ db, int W, const uint32_t* __restrict__ ids,
                                   uint32_t m, uint64_t* __restrict__ out) {
    const uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= uint64_t(m) * W) return;
    const uint32_t i = uint32_t(t / W), w = uint32_t(t - uint64_t(i) * W);
    out[t] = db[uint64_t(ids[i]) * W + w];
}

void widen_u8(const uint8_t* in, uint32_t* out, uint32_t n, cudaStream_t s) {
    if (!n) return;
    widen_u8_kernel<<<grid_for(n, 256), 256, 0, s>>>(in, out, n);
    CURC_LAUNCH_CHECK();
}

void nonzero_u8(const uint8_t* in, uint8_t* out, uint32_t n, cudaStream_t s) {
    if (!n) return;
    nonzero_u8_kernel<<<grid_for(n, 256), 256, 0, s>>>(in, out, n);
    CURC_LAUNCH_CHECK();
}

}  // namespace

void gather_packed_rows(const uint64_t* db, int W, const uint32_t* ids, uint32_t m, uint64_t* out, cudaStream_t s) {
    if (!m) return;
    gather_rows_kernel<<<grid_for(uint64_t(m) * W, 256), 256, 0, s>>>(db, W, ids, m, out);
    CURC_LAUNCH_CHECK();
}

void Block::emit(StageTimer& T) {
    cudaStream_t s = stream;
    const int L = p.L, W = p.W;
    const uint32_t tot = U + NN;
    uint32_t* counts = arena.alloc<uint32_t>(8);
    uint32_t* err = arena.alloc<uint32_t>(2);
    CURC_CHECK(cudaMemsetAsync(err, 0, 8, s));

    // ---- mapped records and unmapped lists (compress.cu:524-594)
    T.begin("emit");
    DevRecord* all_map = arena.alloc<DevRecord>(tot ? tot : 1);
    uint8_t* mapped = arena.alloc<uint8_t>(tot ? tot : 1);
    uint8_t* unm_u = arena.alloc<uint8_t>(U ? U : 1);
    uint8_t* unm_n = arena.alloc<uint8_t>(NN ? NN : 1);
    if (tot) {
        map_records_kernel<<<grid_for(tot, 256), 256, 0, s>>>(mo.mm, mo.strand, mo.pos, U, NN, p.max_mm,
                                                              unmatch_ids, mapped, unm_u, unm_n, all_map);
        CURC_LAUNCH_CHECK();
    }
    // records: pseudogenome reads then mapped reads; mismatch counts alongside
    const uint32_t nrec_max = hq.n_records + tot;
    DevRecord* rec = arena.alloc<DevRecord>(nrec_max ? nrec_max : 1);
    uint8_t* mis = arena.alloc<uint8_t>(nrec_max ? nrec_max : 1);
    if (hq.n_records)
        CURC_CHECK(cudaMemcpyAsync(rec, hq.records, size_t(hq.n_records) * sizeof(DevRecord), cudaMemcpyDeviceToDevice, s));
    CURC_CHECK(cudaMemsetAsync(mis, 0, hq.n_records ? hq.n_records : 1, s));
    {
        // compaction of 16-byte records: select their indices, then gather
        uint32_t* sel = arena.alloc<uint32_t>(tot ? tot : 1);
        select_indices(mapped, sel, tot, counts + 0, arena, s);
        const uint32_t nm = read_scalar(counts + 0, s);
        n_map = nm;
        if (nm) {
            gather_records_kernel<<<grid_for(nm, 256), 256, 0, s>>>(all_map, mo.mm, sel, nm, rec + hq.n_records,
                                                                   mis + hq.n_records);
            CURC_LAUNCH_CHECK();
        }
    }
    const uint32_t Tn = hq.n_records + n_map;
    n_records = Tn;
    // unmapped lists
    ug = arena.alloc<uint32_t>(U ? U : 1);
    select_flagged(unmatch_ids, unm_u, ug, U, counts + 1, arena, s);
    un = arena.alloc<uint32_t>(NN ? NN : 1);
    select_indices(unm_n, un, NN, counts + 2, arena, s);
    {
        uint32_t hc[2];
        read_small(hc, counts + 1, 8, s);
        n_ug = hc[0];
        n_un = hc[1];
    }

    // ---- order records (compress.cu:1743-1756)
    srec = arena.alloc<DevRecord>(Tn ? Tn : 1);
    smis = arena.alloc<uint8_t>(Tn ? Tn : 1);
    if (Tn) {
        auto mk = arena.mark();
        uint64_t* key = arena.alloc<uint64_t>(Tn);
        uint32_t* idx = arena.alloc<uint32_t>(Tn);
        sort_keys_kernel<<<grid_for(Tn, 256), 256, 0, s>>>(rec, Tn, p.preserve_order, n_ids, key, idx);
        CURC_LAUNCH_CHECK();
        int bits = 1;
        const uint64_t maxkey = p.preserve_order ? uint64_t(n) : hq.len;
        while (bits < 64 && (1ull << bits) <= maxkey) ++bits;
        radix_sort_pairs<uint64_t, uint32_t>(key, idx, Tn, 0, bits, arena, s);
        gather_records_kernel<<<grid_for(Tn, 256), 256, 0, s>>>(rec, mis, idx, Tn, srec, smis);
        CURC_LAUNCH_CHECK();
        arena.release(mk);
    }

    // ---- per-record streams
    char* strand = arena.alloc<char>(Tn ? Tn : 1);
    uint16_t* read_off = arena.alloc<uint16_t>(Tn ? Tn : 1);
    const uint32_t pe_total = (!p.preserve_order && p.paired_end) ? n : 0;
    pe_order = arena.alloc<uint32_t>(pe_total ? pe_total : 1);
    id_to_pos = arena.alloc<uint64_t>(p.preserve_order ? n : 1);
    if (p.preserve_order && n) fill<uint64_t>(id_to_pos, 0, n, s);
    if (Tn) {
        record_streams_kernel<<<grid_for(Tn, 256), 256, 0, s>>>(srec, Tn, p.preserve_order, p.paired_end, n_ids, strand,
                                                                read_off, pe_order, id_to_pos);
        CURC_LAUNCH_CHECK();
    }

    // ---- mismatches (compress.cu:1815-1886)
    uint32_t* base_idx = arena.alloc<uint32_t>(Tn + 1);
    uint32_t* mis32 = arena.alloc<uint32_t>(Tn + 1);
    CURC_CHECK(cudaMemsetAsync(mis32, 0, size_t(Tn + 1) * 4, s));
    widen_u8(smis, mis32, Tn, s);
    uint32_t* nbases_dev = counts + 3;
    exclusive_scan<uint32_t>(mis32, base_idx, Tn, nbases_dev, arena, s);
    const uint32_t nbases = read_scalar(nbases_dev, s);
    n_mis = nbases;
    mctx = arena.alloc<uint8_t>(nbases ? nbases : 1);
    mbase = arena.alloc<uint8_t>(nbases ? nbases : 1);
    // classes
    const int maxm = p.max_mm;
    uint32_t* chist = arena.alloc<uint32_t>(maxm + 2);
    CURC_CHECK(cudaMemsetAsync(chist, 0, size_t(maxm + 2) * 4, s));
    if (Tn) {
        class_hist_kernel<<<resident_grid(class_hist_kernel, 256, Tn), 256, 0, s>>>(smis, Tn, maxm + 2, chist);
        CURC_LAUNCH_CHECK();
    }
    std::vector<uint32_t> hcls(maxm + 2);
    read_small(hcls.data(), chist, size_t(maxm + 2) * 4, s);
    class_count.assign(maxm + 1, 0);
    std::vector<uint32_t> first(maxm + 2, 0);
    std::vector<uint64_t> cbase(maxm + 2, 0);
    uint32_t acc = 0;
    uint64_t eacc = 0;
    for (int mm = 1; mm <= maxm; ++mm) {
        class_count[mm] = hcls[mm];
        first[mm] = acc;
        cbase[mm] = eacc;
        acc += hcls[mm];
        eacc += uint64_t(hcls[mm]) * class_width(mm);
    }
    class_elems = eacc;
    uint32_t* d_first = arena.alloc<uint32_t>(maxm + 2);
    uint64_t* d_cbase = arena.alloc<uint64_t>(maxm + 2);
    CURC_CHECK(cudaMemcpyAsync(d_first, first.data(), size_t(maxm + 2) * 4, cudaMemcpyHostToDevice, s));
    CURC_CHECK(cudaMemcpyAsync(d_cbase, cbase.data(), size_t(maxm + 2) * 8, cudaMemcpyHostToDevice, s));
    uint32_t* crank = arena.alloc<uint32_t>(Tn ? Tn : 1);
    off_all = arena.alloc<uint16_t>(eacc ? eacc : 1);
    if (acc) {
        auto mk = arena.mark();
        uint8_t* has = arena.alloc<uint8_t>(Tn);
        nonzero_u8(smis, has, Tn, s);
        uint32_t* sel = arena.alloc<uint32_t>(acc);
        select_indices(has, sel, Tn, counts + 4, arena, s);
        uint32_t* key = arena.alloc<uint32_t>(acc);
        class_keys_kernel<<<grid_for(acc, 256), 256, 0, s>>>(sel, acc, smis, key);
        CURC_LAUNCH_CHECK();
        radix_sort_pairs<uint32_t, uint32_t>(key, sel, acc, 0, 8, arena, s);
        class_rank_kernel<<<grid_for(acc, 256), 256, 0, s>>>(key, sel, acc, d_first, crank);
        CURC_LAUNCH_CHECK();
        arena.release(mk);
        EmitCtx e{srec, smis, base_idx, crank, d_cbase, db, nreads, hq.seq, hq.packed, L, W, mctx, mbase, off_all, err};
        mismatch_kernel<<<grid_for(Tn, 128), 128, 0, s>>>(e, Tn);
        CURC_LAUNCH_CHECK();
    }
    // context recode (compress.cu:1889-1929)
    unsigned long long* chh = arena.alloc<unsigned long long>(20);
    CURC_CHECK(cudaMemsetAsync(chh, 0, 20 * 8, s));
    uint8_t* rank = arena.alloc<uint8_t>(20);
    char* table = arena.alloc<char>(16);
    if (nbases) {
        ctx_hist_kernel<<<grid_for(nbases, 256, 8), 256, 0, s>>>(mctx, mbase, nbases, chh, err);
        CURC_LAUNCH_CHECK();
    }
    ctx_rank_kernel<<<1, 32, 0, s>>>(chh, rank, table);
    CURC_LAUNCH_CHECK();
    if (nbases) {
        recode_kernel<<<grid_for(nbases, 256, 8), 256, 0, s>>>(mctx, mbase, nbases, rank);
        CURC_LAUNCH_CHECK();
    }
    {
        uint32_t he[2];
        read_small(he, err, 8, s);
        if (he[0]) throw std::runtime_error("emit: mismatch count disagrees with mapping");
        if (he[1]) throw std::runtime_error("emit: unexpected symbol in a mismatch");
    }
    T.end();

    // ---- a11: unmapped pseudogenomes (compress.cu:1649-1728)
    T.begin("unmapped_refs");
    if (n_ug) {
        uint64_t* ldb = arena.alloc<uint64_t>(size_t(n_ug) * W + 1);
        gather_packed_rows(db, W, ug, n_ug, ldb, s);
        uint32_t* nx = arena.alloc<uint32_t>(n_ug);
        uint32_t* pv = arena.alloc<uint32_t>(n_ug);
        uint16_t* of = arena.alloc<uint16_t>(n_ug);
        fill<uint32_t>(nx, INVALID, n_ug, s);
        fill<uint32_t>(pv, INVALID, n_ug, s);
        fill<uint16_t>(of, INVALOFF, n_ug, s);
        uint32_t* seqids = arena.alloc<uint32_t>(n_ug);
        iota(seqids, n_ug, s);
        {
            auto mk = arena.mark();
            uint32_t* pre = arena.alloc<uint32_t>(n_ug);
            uint32_t* suf = arena.alloc<uint32_t>(n_ug);
            iota(pre, n_ug, s);
            iota(suf, n_ug, s);
            full_match_packed(p, ldb, pre, suf, n_ug, nx, pv, of, arena, s);
            arena.release(mk);
        }
        assemble(ldb, nullptr, L, W, seqids, n_ug, n_ug, nx, pv, of, false, lq, arena, s);
    } else {
        lq = Assembled{};
        lq.records = arena.alloc<DevRecord>(1);
        lq.seq = arena.alloc<uint8_t>(1);
        lq.packed = arena.alloc<uint64_t>(1);
        CURC_CHECK(cudaMemsetAsync(lq.packed, 0, 8, s));
    }
    if (n_un) {
        uint32_t* nx = arena.alloc<uint32_t>(NN);
        uint32_t* pv = arena.alloc<uint32_t>(NN);
        uint16_t* of = arena.alloc<uint16_t>(NN);
        full_match_ascii(p, nreads, un, n_un, NN, nx, pv, of, arena, s);  // sorts `un`
        assemble(nullptr, nreads, L, W, un, n_un, NN, nx, pv, of, true, lqn, arena, s);
    } else {
        lqn = Assembled{};
        lqn.records = arena.alloc<DevRecord>(1);
        lqn.seq = arena.alloc<uint8_t>(1);
        lqn.packed = arena.alloc<uint64_t>(1);
        CURC_CHECK(cudaMemsetAsync(lqn.packed, 0, 8, s));
    }
    // offsets / order / positions of unmapped reads (compress.cu:1964-2006)
    uint16_t* uoff = arena.alloc<uint16_t>(lq.n_records ? lq.n_records : 1);
    uint16_t* unoff = arena.alloc<uint16_t>(lqn.n_records ? lqn.n_records : 1);
    if (lq.n_records) {
        unmapped_offsets_kernel<<<grid_for(lq.n_records, 256), 256, 0, s>>>(
            lq.records, lq.n_records, L, p.preserve_order, p.paired_end, ug, hq.len, uoff, pe_order + Tn, id_to_pos);
        CURC_LAUNCH_CHECK();
    }
    if (lqn.n_records) {
        unmapped_offsets_kernel<<<grid_for(lqn.n_records, 256), 256, 0, s>>>(
            lqn.records, lqn.n_records, L, p.preserve_order, p.paired_end, n_ids, hq.len + lq.len, unoff,
            pe_order + Tn + lq.n_records, id_to_pos);
        CURC_LAUNCH_CHECK();
    }
    T.end();

    // ---- host copies of the streams
    keep("strand", strand, Tn);
    keep("mis_cnt", smis, Tn);
    keep("mis_base", mbase, nbases);
    keep("decoder_table", table, 16);
    if (!p.preserve_order) {
        keep("read_off", read_off, Tn);
        keep("unmap_read_off", uoff, lq.n_records);
        keep("unmap_n_read_off", unoff, lqn.n_records);
        keep("pe_order", pe_order, pe_total);
        keep("id_to_pos", id_to_pos, 0);
    } else {
        keep("read_off", read_off, 0);
        keep("unmap_read_off", uoff, 0);
        keep("unmap_n_read_off", unoff, 0);
        keep("pe_order", pe_order, 0);
        keep("id_to_pos", id_to_pos, n);
    }
    {
        // per-class offset streams: consecutive slices of off_all
        uint64_t b = 0;
        for (int mm = 1; mm <= p.max_mm; ++mm) {
            const uint64_t ne = uint64_t(class_count[mm]) * class_width(mm);
            keep("mis_off_" + std::to_string(mm), off_all + b, ne);
            b += ne;
        }
    }
    if (keep_intermediates) {
        keep("unmap_seq", lq.seq, lq.len);
        keep("unmap_n_seq", lqn.seq, lqn.len);
    }

    // ---- a12: reverse-complement repeat removal
    T.begin("refmatch");
    refmatch_all();
    T.end();
}

}  // namespace curc
