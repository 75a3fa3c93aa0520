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
// B200 design: list ranking by pointer jumping (at most log2 rounds, double
// buffered, 32-byte state per read so a jump is one sector) gives each read
// its chain head, base offset and rank; cycles are found as reads whose
// ancestor pointer never clears and are cut in parallel (below); chains are
// ordered by (min list index) with a radix sort and placed by exclusive
// scans; every read then writes its bases independently.
#include "stages.cuh"

namespace curc {

namespace {

__global__ void scatter_index_kernel(const uint32_t* __restrict__ ids, uint32_t m, uint32_t* __restrict__ pos_in_ids) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) pos_in_ids[ids[i]] = i;
}

// Pointer-jumping state of one read, 32 bytes so that one jump gathers one
// sector.
struct __align__(32) RankState {
    uint64_t acc;     // bases contributed by the reads before this one (so far)
    uint32_t jump;    // ancestor 2^t links back, INVALID once past the head
    uint32_t far;     // farthest ancestor reached (the head at convergence)
    uint32_t cnt;     // reads before this one (so far)
    uint32_t mn;      // smallest list index over the reads covered
    uint32_t member;  // read belongs to this assembly
    uint32_t pad;
};

// Reads are processed in id order so that a read's own state is read and
// written coalesced; only the ancestor's state is a random gather.
__global__ void rank_init_kernel(uint32_t n, const uint32_t* __restrict__ pv, const uint16_t* __restrict__ offset,
                                 const uint32_t* __restrict__ pos_in_ids, const uint8_t* __restrict__ redo,
                                 const RankState* __restrict__ keep, RankState* __restrict__ out) {
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= n) return;
    if (redo && !redo[x]) {
        out[x] = keep[x];
        return;
    }
    RankState st;
    st.pad = 0;
    st.member = pos_in_ids[x] != INVALID;
    const uint32_t p = st.member ? pv[x] : INVALID;
    st.jump = p;
    st.far = p == INVALID ? x : p;
    st.acc = p == INVALID ? 0 : offset[p];
    st.cnt = p == INVALID ? 0 : 1;
    st.mn = pos_in_ids[x];
    out[x] = st;
}

// One jump for every read (grid-stride); *active counts the reads whose
// ancestor pointer is still set afterwards.
__global__ void __launch_bounds__(512) rank_step_kernel(uint32_t n, const RankState* __restrict__ in,
                                                        RankState* __restrict__ out, uint32_t* __restrict__ active) {
    uint32_t still = 0;
    for (uint32_t x = blockIdx.x * blockDim.x + threadIdx.x; x < n; x += gridDim.x * blockDim.x) {
        RankState st = in[x];
        if (st.jump != INVALID) {
            const RankState a = in[st.jump];
            st.far = a.far;
            st.acc += a.acc;
            st.cnt += a.cnt;
            st.mn = min(st.mn, a.mn);
            st.jump = a.jump;
            still += st.jump != INVALID;
        }
        out[x] = st;
    }
    block_tally<uint32_t>(still, active);
}

__global__ void cycle_flags_kernel(uint32_t n, const RankState* __restrict__ st, uint8_t* __restrict__ cyc) {
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x < n) cyc[x] = st[x].member && st[x].jump != INVALID;
}

// Cycles are cut in parallel.  The reference walks each cycle from the
// successor h of its first listed read r (the read visited first) round to
// r, and cuts after the first read of largest offset met on the way.  Here:
// (1) a temporary cut before h makes each cycle a chain h .. r;
// (2) ranking that chain gives every read its walk position;
// (3) the largest (offset, -position) over the chain picks the cut read;
// (4) the temporary cut is undone and the real one made.

// (1) r = the cycle read whose list index is the cycle's minimum.
__global__ void cycle_open_kernel(uint32_t n, const RankState* __restrict__ st, const uint8_t* __restrict__ cyc,
                                  const uint32_t* __restrict__ pos_in_ids, const uint32_t* __restrict__ nx,
                                  uint32_t* pv, uint32_t* __restrict__ leader_of_head, uint32_t* __restrict__ err) {
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= n || !cyc[x] || st[x].mn != pos_in_ids[x]) return;
    const uint32_t h = nx[x];
    if (h == INVALID || pv[h] != x) {
        atomicExch(err, 1u);
        return;
    }
    leader_of_head[h] = x;
    pv[h] = INVALID;
}

// (3) per chain head: max of (offset << 32 | ~position)
__global__ void cycle_max_kernel(uint32_t n, const RankState* __restrict__ st, const uint8_t* __restrict__ cyc,
                                 const uint16_t* __restrict__ offset, unsigned long long* __restrict__ best) {
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= n || !cyc[x]) return;
    const unsigned long long key = (unsigned long long)offset[x] << 32 | (0xFFFFFFFFu - st[x].cnt);
    atomicMax(&best[st[x].far], key);
}

// (4) the read that holds its chain's maximum restores the temporary cut and
// makes the real one after itself.
__global__ void cycle_cut_kernel(uint32_t n, const RankState* __restrict__ st, const uint8_t* __restrict__ cyc,
                                 const unsigned long long* __restrict__ best,
                                 const uint32_t* __restrict__ leader_of_head, uint32_t* nx, uint32_t* pv) {
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= n || !cyc[x]) return;
    const uint32_t h = st[x].far;
    if ((0xFFFFFFFFu - uint32_t(best[h] & 0xFFFFFFFFull)) != st[x].cnt) return;
    pv[h] = leader_of_head[h];
    const uint32_t nh = nx[x];
    nx[x] = INVALID;
    pv[nh] = INVALID;
}

__global__ void chain_key_kernel(uint32_t n, const RankState* __restrict__ st, uint32_t* __restrict__ key) {
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    // mn covers the read and its predecessors, so the minimum over the
    // chain's reads is the chain's first list index
    if (x < n && st[x].member) atomicMin(&key[st[x].far], st[x].mn);
}

__global__ void head_flags_kernel(const uint32_t* __restrict__ ids, uint32_t m, const uint32_t* __restrict__ pv,
                                  uint8_t* __restrict__ f) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) f[i] = pv[ids[i]] == INVALID;
}

__global__ void tail_sizes_kernel(uint32_t n, const uint32_t* __restrict__ nx, const RankState* __restrict__ st,
                                  int L, uint64_t* __restrict__ chain_bases, uint32_t* __restrict__ chain_members) {
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= n || !st[x].member || nx[x] != INVALID) return;
    chain_bases[st[x].far] = st[x].acc + uint64_t(L);
    chain_members[st[x].far] = st[x].cnt + 1;
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

__global__ void place_kernel(const uint32_t* __restrict__ ids, uint32_t m, const uint32_t* __restrict__ nx,
                             const RankState* __restrict__ st,
                             const uint32_t* __restrict__ slot, const uint64_t* __restrict__ cpos,
                             const uint32_t* __restrict__ crec, const uint16_t* __restrict__ offset,
                             const uint64_t* __restrict__ db, const uint8_t* __restrict__ ascii, int L, int W,
                             uint8_t is_n, DevRecord* __restrict__ rec, uint8_t* __restrict__ seq) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const uint32_t x = ids[i];
    const RankState r = st[x];
    const uint32_t c = slot[r.far];
    const uint64_t pos = cpos[c] + r.acc;
    DevRecord d;
    d.read_id = x;
    d.is_n = is_n;
    d.strand = 0;
    d.pad = 0;
    d.pos = pos;
    rec[crec[c] + r.cnt] = d;
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

// Pointer jumping to convergence (early exit when no pointer is left, at
// most enough rounds for a chain of every member).  Returns the final state
// and, in *left, the number of reads whose pointer never cleared (cycles).
RankState* run_ranking(uint32_t n, uint32_t m, const uint32_t* pv, const uint16_t* offset, const uint32_t* pos_in_ids,
                       const uint8_t* redo, const RankState* keep, RankState* A, RankState* B, uint32_t* active,
                       uint32_t* left, cudaStream_t s) {
    const int g = grid_for(n, 256);
    rank_init_kernel<<<g, 256, 0, s>>>(n, pv, offset, pos_in_ids, redo, keep, A);
    CURC_LAUNCH_CHECK();
    const int R = rounds_for(m);
    *left = 0;
    for (int t = 0; t < R; ++t) {
        CURC_CHECK(cudaMemsetAsync(active, 0, 4, s));
        rank_step_kernel<<<resident_grid(rank_step_kernel, 512, n), 512, 0, s>>>(n, A, B, active);
        CURC_LAUNCH_CHECK();
        std::swap(A, B);
        *left = read_scalar(active, s);
        if (*left == 0) break;
    }
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
    fill<uint32_t>(pos_in_ids, INVALID, n, s);
    scatter_index_kernel<<<g, 256, 0, s>>>(ids, m, pos_in_ids);
    CURC_LAUNCH_CHECK();
    RankState* A = a.alloc<RankState>(n);
    RankState* B = a.alloc<RankState>(n);
    uint32_t* active = a.alloc<uint32_t>(4);
    uint32_t left = 0;
    SubStage sp_rank("assembly.ranking");
    RankState* R = run_ranking(n_total, m, pv, offset, pos_in_ids, nullptr, nullptr, A, B, active, &left, s);
    if (left) {
        // cycles: cut each in parallel, then rank its reads again (the other
        // reads keep their final state from the first ranking)
        const int gn = grid_for(n, 256);
        uint8_t* cyc = a.alloc<uint8_t>(n);
        cycle_flags_kernel<<<gn, 256, 0, s>>>(n_total, R, cyc);
        CURC_LAUNCH_CHECK();
        uint32_t* leader_of_head = a.alloc<uint32_t>(n);
        unsigned long long* best = a.alloc<unsigned long long>(n);
        CURC_CHECK(cudaMemsetAsync(best, 0, n * sizeof(unsigned long long), s));
        CURC_CHECK(cudaMemsetAsync(active + 1, 0, 4, s));
        cycle_open_kernel<<<gn, 256, 0, s>>>(n_total, R, cyc, pos_in_ids, nx, pv, leader_of_head, active + 1);
        CURC_LAUNCH_CHECK();
        if (read_scalar(active + 1, s)) throw std::runtime_error("assemble: broken cycle");
        RankState* keep = R;
        RankState* X = keep == A ? B : A;
        RankState* Y = a.alloc<RankState>(n);
        RankState* T = run_ranking(n_total, m, pv, offset, pos_in_ids, cyc, keep, X, Y, active, &left, s);
        if (left) throw std::runtime_error("assemble: cycle still closed after its temporary cut");
        cycle_max_kernel<<<gn, 256, 0, s>>>(n_total, T, cyc, offset, best);
        CURC_LAUNCH_CHECK();
        cycle_cut_kernel<<<gn, 256, 0, s>>>(n_total, T, cyc, best, leader_of_head, nx, pv);
        CURC_LAUNCH_CHECK();
        R = run_ranking(n_total, m, pv, offset, pos_in_ids, cyc, keep, X, Y, active, &left, s);
        if (left) throw std::runtime_error("assemble: unresolved chain links after cutting cycles");
    }
    sp_rank.stop();
    SubStage sp_place("assembly.order_place");
    // chain order: first member in list order
    uint32_t* key = a.alloc<uint32_t>(n);
    fill<uint32_t>(key, INVALID, n, s);
    chain_key_kernel<<<grid_for(n, 256), 256, 0, s>>>(n_total, R, key);
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
    tail_sizes_kernel<<<grid_for(n, 256), 256, 0, s>>>(n_total, nx, R, L, chain_bases, chain_members);
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
