// a8: walk linked reads into a pseudogenome.
//
// Reference: RefRecord::assembly compress.cu:107-217 (a sequential pointer
// chase on the host) and compute_binary_ref compress.cu:229-246.
//
// Output order of the reference: chains in order of their first member in
// the id list; each chain from its head, every read contributing offset[r]
// bases and the tail all L bases; a cycle is cut after its member with the
// largest offset (first maximum met walking from the successor of the
// cycle's first listed member), which becomes the tail.
//
// B200 design: list ranking by pointer jumping (log2 rounds over the member
// set, double buffered) gives each read its chain head, base offset and
// rank; cycles are found as members whose ancestor pointer never clears and
// are cut by one thread each; chains are ordered by (min list index) with a
// radix sort and placed by exclusive scans; every read then writes its
// bases independently.
#include "stages.cuh"

namespace curc {

namespace {

__global__ void scatter_index_kernel(const uint32_t* __restrict__ ids, uint32_t m, uint32_t* __restrict__ pos_in_ids) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) pos_in_ids[ids[i]] = i;
}

struct Rank {
    uint32_t* jump;
    uint32_t* far;
    uint64_t* acc;
    uint32_t* cnt;
    uint32_t* mn;
};

__global__ void rank_init_kernel(const uint32_t* __restrict__ ids, uint32_t m, const uint32_t* __restrict__ pv,
                                 const uint16_t* __restrict__ offset, const uint32_t* __restrict__ pos_in_ids, Rank r) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const uint32_t x = ids[i];
    const uint32_t p = pv[x];
    r.jump[x] = p;
    r.far[x] = p == INVALID ? x : p;
    r.acc[x] = p == INVALID ? 0 : offset[p];
    r.cnt[x] = p == INVALID ? 0 : 1;
    r.mn[x] = pos_in_ids[x];
}

__global__ void rank_step_kernel(const uint32_t* __restrict__ ids, uint32_t m, Rank in, Rank out,
                                 uint32_t* __restrict__ unresolved) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const uint32_t x = ids[i];
    const uint32_t j = in.jump[x];
    if (j == INVALID) {
        out.jump[x] = INVALID;
        out.far[x] = in.far[x];
        out.acc[x] = in.acc[x];
        out.cnt[x] = in.cnt[x];
        out.mn[x] = in.mn[x];
        return;
    }
    out.far[x] = in.far[j];
    out.acc[x] = in.acc[x] + in.acc[j];
    out.cnt[x] = in.cnt[x] + in.cnt[j];
    out.mn[x] = min(in.mn[x], in.mn[j]);
    const uint32_t jj = in.jump[j];
    out.jump[x] = jj;
    if (unresolved && jj != INVALID) atomicAdd(unresolved, 1u);
}

// One thread per cycle (its first listed member): cut after the first
// maximum-offset member met walking from that member's successor.
__global__ void cut_cycles_kernel(const uint32_t* __restrict__ ids, uint32_t m, Rank r,
                                  const uint32_t* __restrict__ pos_in_ids, const uint16_t* __restrict__ offset,
                                  uint32_t* nx, uint32_t* pv, uint32_t* __restrict__ err) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const uint32_t x = ids[i];
    if (r.jump[x] == INVALID || r.mn[x] != pos_in_ids[x]) return;
    uint32_t c = nx[x];
    if (c == INVALID) {
        atomicExch(err, 1u);
        return;
    }
    uint16_t mo = offset[c];
    uint32_t mid = c;
    uint32_t steps = 0;
    while (c != x) {
        c = nx[c];
        if (c == INVALID || ++steps > m) {  // not a cycle: report, touch nothing
            atomicExch(err, 1u);
            return;
        }
        if (offset[c] > mo) {
            mo = offset[c];
            mid = c;
        }
    }
    const uint32_t h = nx[mid];
    nx[mid] = INVALID;
    pv[h] = INVALID;
}

__global__ void chain_key_kernel(const uint32_t* __restrict__ ids, uint32_t m, const uint32_t* __restrict__ far,
                                 uint32_t* __restrict__ key) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) atomicMin(&key[far[ids[i]]], i);
}

__global__ void head_flags_kernel(const uint32_t* __restrict__ ids, uint32_t m, const uint32_t* __restrict__ pv,
                                  uint8_t* __restrict__ f) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) f[i] = pv[ids[i]] == INVALID;
}

__global__ void tail_sizes_kernel(const uint32_t* __restrict__ ids, uint32_t m, const uint32_t* __restrict__ nx, Rank r,
                                  int L, uint64_t* __restrict__ chain_bases, uint32_t* __restrict__ chain_members) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const uint32_t x = ids[i];
    if (nx[x] != INVALID) return;
    chain_bases[r.far[x]] = r.acc[x] + uint64_t(L);
    chain_members[r.far[x]] = r.cnt[x] + 1;
}

__global__ void gather_heads_kernel(const uint32_t* __restrict__ heads, uint32_t nh, const uint32_t* __restrict__ key,
                                    uint32_t* __restrict__ hkey) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < nh) hkey[t] = key[heads[t]];
}

__global__ void chain_sizes_sorted_kernel(const uint32_t* __restrict__ heads, uint32_t nh,
                                          const uint64_t* __restrict__ chain_bases,
                                          const uint32_t* __restrict__ chain_members, uint64_t* __restrict__ cb,
                                          uint32_t* __restrict__ cm, uint32_t* __restrict__ slot) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nh) return;
    const uint32_t h = heads[t];
    cb[t] = chain_bases[h];
    cm[t] = chain_members[h];
    slot[h] = t;
}

__global__ void place_kernel(const uint32_t* __restrict__ ids, uint32_t m, const uint32_t* __restrict__ nx, Rank r,
                             const uint32_t* __restrict__ slot, const uint64_t* __restrict__ cpos,
                             const uint32_t* __restrict__ crec, const uint16_t* __restrict__ offset,
                             const uint64_t* __restrict__ db, const uint8_t* __restrict__ ascii, int L, int W,
                             uint8_t is_n, DevRecord* __restrict__ rec, uint8_t* __restrict__ seq) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const uint32_t x = ids[i];
    const uint32_t c = slot[r.far[x]];
    const uint64_t pos = cpos[c] + r.acc[x];
    DevRecord d;
    d.read_id = x;
    d.is_n = is_n;
    d.strand = 0;
    d.pad = 0;
    d.pos = pos;
    rec[crec[c] + r.cnt[x]] = d;
    const int nb = nx[x] == INVALID ? L : offset[x];
    uint8_t* out = seq + pos;
    if (ascii) {
        const uint8_t* src = ascii + uint64_t(x) * L;
        for (int j = 0; j < nb; ++j) out[j] = src[j];
    } else {
        const uint64_t* rd = db + uint64_t(x) * W;
        for (int j = 0; j < nb; ++j) out[j] = "ACGT"[code_at(rd, j)];
    }
}

__global__ void pack_ref_kernel(const uint8_t* __restrict__ seq, uint64_t len, uint64_t* __restrict__ packed,
                                uint64_t words) {
    for (uint64_t w = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; w < words; w += uint64_t(gridDim.x) * blockDim.x) {
        uint64_t v = 0;
        const uint64_t b = w * 32;
        for (int j = 0; j < 32; ++j) {
            const uint64_t q = b + j;
            v = (v << 2) | uint64_t(q < len ? ascii_code(seq[q]) : 0);
        }
        packed[w] = v;
    }
}

inline int rounds_for(uint32_t m) {
    int r = 1;
    while ((1ull << r) < uint64_t(m) + 1) ++r;
    return r + 1;
}

Rank alloc_rank(uint32_t n, Arena& a) {
    return Rank{a.alloc<uint32_t>(n), a.alloc<uint32_t>(n), a.alloc<uint64_t>(n), a.alloc<uint32_t>(n),
                a.alloc<uint32_t>(n)};
}

// Runs pointer jumping to convergence; returns the final buffer and the
// number of members whose ancestor pointer is still set (cycle members).
Rank run_ranking(const uint32_t* ids, uint32_t m, const uint32_t* pv, const uint16_t* offset,
                 const uint32_t* pos_in_ids, Rank A, Rank B, uint32_t* unresolved, uint32_t* n_unresolved,
                 cudaStream_t s) {
    const int g = grid_for(m, 256);
    rank_init_kernel<<<g, 256, 0, s>>>(ids, m, pv, offset, pos_in_ids, A);
    CURC_LAUNCH_CHECK();
    const int R = rounds_for(m);
    for (int t = 0; t < R; ++t) {
        const bool last = t == R - 1;
        if (last) CURC_CHECK(cudaMemsetAsync(unresolved, 0, 4, s));
        rank_step_kernel<<<g, 256, 0, s>>>(ids, m, A, B, last ? unresolved : nullptr);
        CURC_LAUNCH_CHECK();
        std::swap(A, B);
    }
    *n_unresolved = read_scalar(unresolved, s);
    return A;
}

}  // namespace

void pack_ascii_ref(const uint8_t* seq, uint64_t len, uint64_t* packed, cudaStream_t s) {
    const uint64_t words = (len + 31) / 32 + 1;
    pack_ref_kernel<<<grid_for(words, 256), 256, 0, s>>>(seq, len, packed, words);
    CURC_LAUNCH_CHECK();
}

void assemble(const uint64_t* db, const uint8_t* ascii, int L, int W, const uint32_t* ids, uint32_t m,
              uint32_t n_total, const uint32_t* next, const uint32_t* prev, const uint16_t* offset, bool is_n,
              Assembled& out, Arena& a, cudaStream_t s) {
    out.n_records = m;
    out.records = a.alloc<DevRecord>(m ? m : 1);
    if (m == 0) {
        out.len = 0;
        out.seq = a.alloc<uint8_t>(1);
        out.packed = a.alloc<uint64_t>(1);
        CURC_CHECK(cudaMemsetAsync(out.packed, 0, 8, s));
        return;
    }
    const size_t n = n_total;
    uint32_t* pos_in_ids = a.alloc<uint32_t>(n);
    uint32_t* nx = a.alloc<uint32_t>(n);
    uint32_t* pv = a.alloc<uint32_t>(n);
    CURC_CHECK(cudaMemcpyAsync(nx, next, n * 4, cudaMemcpyDeviceToDevice, s));
    CURC_CHECK(cudaMemcpyAsync(pv, prev, n * 4, cudaMemcpyDeviceToDevice, s));
    const int g = grid_for(m, 256);
    scatter_index_kernel<<<g, 256, 0, s>>>(ids, m, pos_in_ids);
    CURC_LAUNCH_CHECK();
    Rank A = alloc_rank(n_total, a), B = alloc_rank(n_total, a);
    fill<uint32_t>(A.jump, INVALID, n, s);
    fill<uint32_t>(B.jump, INVALID, n, s);
    fill<uint32_t>(A.far, INVALID, n, s);
    fill<uint32_t>(B.far, INVALID, n, s);
    uint32_t* unresolved = a.alloc<uint32_t>(4);
    uint32_t nun = 0;
    Rank R = run_ranking(ids, m, pv, offset, pos_in_ids, A, B, unresolved, &nun, s);
    if (nun) {
        CURC_CHECK(cudaMemsetAsync(unresolved + 1, 0, 4, s));
        cut_cycles_kernel<<<g, 256, 0, s>>>(ids, m, R, pos_in_ids, offset, nx, pv, unresolved + 1);
        CURC_LAUNCH_CHECK();
        if (read_scalar(unresolved + 1, s)) throw std::runtime_error("assemble: broken chain while cutting cycles");
        R = run_ranking(ids, m, pv, offset, pos_in_ids, A, B, unresolved, &nun, s);
        if (nun) throw std::runtime_error("assemble: unresolved chain links after cutting cycles");
    }
    // chain order: first member in list order
    uint32_t* key = a.alloc<uint32_t>(n);
    fill<uint32_t>(key, INVALID, n, s);
    chain_key_kernel<<<g, 256, 0, s>>>(ids, m, R.far, key);
    CURC_LAUNCH_CHECK();
    uint8_t* hf = a.alloc<uint8_t>(m);
    head_flags_kernel<<<g, 256, 0, s>>>(ids, m, pv, hf);
    CURC_LAUNCH_CHECK();
    uint32_t* heads = a.alloc<uint32_t>(m);
    uint32_t* cnt = a.alloc<uint32_t>(2);
    select_flagged(ids, hf, heads, m, cnt, a, s);
    const uint32_t nh = read_scalar(cnt, s);
    uint32_t* hkey = a.alloc<uint32_t>(nh);
    gather_heads_kernel<<<grid_for(nh, 256), 256, 0, s>>>(heads, nh, key, hkey);
    CURC_LAUNCH_CHECK();
    radix_sort_pairs<uint32_t, uint32_t>(hkey, heads, nh, 0, 32, a, s);
    uint64_t* chain_bases = a.alloc<uint64_t>(n);
    uint32_t* chain_members = a.alloc<uint32_t>(n);
    tail_sizes_kernel<<<g, 256, 0, s>>>(ids, m, nx, R, L, chain_bases, chain_members);
    CURC_LAUNCH_CHECK();
    uint64_t* cpos = a.alloc<uint64_t>(nh + 1);
    uint32_t* crec = a.alloc<uint32_t>(nh + 1);
    uint32_t* slot = a.alloc<uint32_t>(n);
    chain_sizes_sorted_kernel<<<grid_for(nh, 256), 256, 0, s>>>(heads, nh, chain_bases, chain_members, cpos, crec,
                                                                 slot);
    CURC_LAUNCH_CHECK();
    uint64_t* total = a.alloc<uint64_t>(1);
    exclusive_scan<uint64_t>(cpos, cpos, nh, total, a, s);
    exclusive_scan<uint32_t>(crec, crec, nh, cnt + 1, a, s);
    out.len = read_scalar(total, s);
    out.seq = a.alloc<uint8_t>(out.len + 64);
    place_kernel<<<g, 256, 0, s>>>(ids, m, nx, R, slot, cpos, crec, offset, db, ascii, L, W, is_n ? 1 : 0,
                                   out.records, out.seq);
    CURC_LAUNCH_CHECK();
    out.packed = a.alloc<uint64_t>((out.len + 31) / 32 + 1);
    pack_ascii_ref(out.seq, out.len, out.packed, s);
}

}  // namespace curc
