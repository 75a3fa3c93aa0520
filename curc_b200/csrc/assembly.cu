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
// B200 design: list ranking with a sparse ruling set.  Every chain head and
// one member in 8 (by a hash of its id) is a ruler; one thread per ruler
// walks its sublist up to the next ruler, giving every read its offset
// within the sublist; the rulers (about an eighth of the reads, resident
// in L2) are then ranked by pointer jumping, and one pass over the members
// adds the two.  Each read is touched a constant number of times instead of
// once per jumping round.  Cycles show up as ruler lists whose pointers never
// clear (a cycle without any ruler gets one: its member of smallest list
// index) and are cut in parallel (below); chains are ordered by their first
// list index with a radix sort and placed by exclusive scans; every read
// then writes its bases independently.
#include "stages.cuh"

namespace curc {

namespace {

__global__ void scatter_index_kernel(const uint32_t* __restrict__ ids, uint32_t m, uint32_t* __restrict__ pos_in_ids) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) pos_in_ids[ids[i]] = i;
}

constexpr uint32_t RULER_SPACING = 8;  // one sampled ruler per 8 members (power of two)

// Pointer-jumping state, 32 bytes so that one jump gathers one sector.  For
// a ruler: acc / cnt = bases / reads of the sublists before its own, mn = the
// smallest list index over its own and the preceding sublists, far = the
// chain's head ruler.  The final per-member state (indexed by list index)
// has the same fields for the read itself: far = the head read, acc = its
// base offset in the chain, cnt = its rank, and mn, which covers at least
// the read's predecessors and is the chain's (or cycle's) minimum at the
// tail (or on a cycle).
struct __align__(32) RankState {
    uint64_t acc;
    uint32_t jump;    // ruler 2^t sublists back, INVALID once past the head
    uint32_t far;
    uint32_t cnt;
    uint32_t mn;
    uint32_t pad0, pad1;
};

// The links of one read in one 16-byte gather: successor, the read's own
// offset to it, list index, ruler index (INVALID unless a ruler).
struct __align__(16) ChainNode {
    uint32_t nx, off, pos, rix;
};

// Position of a read within its ruler's sublist (indexed by list index).
struct __align__(32) SubPos {
    uint64_t la;     // bases from the ruler's first base to this read's
    uint32_t owner;  // ruler index
    uint32_t lc;     // reads between the ruler and this read
    uint32_t lm;     // smallest list index from the ruler to this read
    uint32_t epoch;  // walk that wrote the entry; older entries mean "not reached"
    uint32_t pad1, pad2;
};

// Totals of one ruler's sublist.
struct __align__(16) SubTotal {
    uint64_t acc;   // bases from the ruler's first base to the next ruler's
    uint32_t cnt;   // reads in the sublist
    uint32_t mn;    // smallest list index in the sublist
};

__global__ void ruler_flags_kernel(const uint32_t* __restrict__ ids, uint32_t m, const uint32_t* __restrict__ pv,
                                   const uint8_t* __restrict__ promote, uint8_t* __restrict__ f) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const uint32_t x = ids[i];
    f[i] = pv[x] == INVALID || (murmur64(x) & (RULER_SPACING - 1)) == 0 || (promote && promote[i]);
}

// One node per read, written in read order (non-members get INVALID
// fields, so a link out of the member set is caught by the walk).
__global__ void chain_nodes_kernel(uint32_t n, const uint32_t* __restrict__ pos_in_ids,
                                   const uint32_t* __restrict__ nx, const uint16_t* __restrict__ offset,
                                   ChainNode* __restrict__ node) {
    for (uint32_t x = blockIdx.x * blockDim.x + threadIdx.x; x < n; x += gridDim.x * blockDim.x) {
        const uint32_t i = pos_in_ids[x];
        if (i == INVALID) {
            node[x] = ChainNode{INVALID, 0u, INVALID, INVALID};
        } else {
            const uint32_t nn = nx[x];
            node[x] = ChainNode{nn, nn == INVALID ? 0u : uint32_t(offset[x]), i, INVALID};
        }
    }
}

__global__ void ruler_index_kernel(const uint32_t* __restrict__ rul, uint32_t nr, ChainNode* __restrict__ node) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < nr) node[rul[t]].rix = t;
}

// One thread per ruler walks its sublist; the walk ends at the next ruler
// or the chain's tail (a walk that comes back to a ruler on a cycle ends
// there too), at most m steps.
__global__ void ruler_walk_kernel(const uint32_t* __restrict__ rul, uint32_t nr, uint32_t m, uint32_t n,
                                  uint32_t epoch, const ChainNode* __restrict__ node, SubPos* __restrict__ loc,
                                  SubTotal* __restrict__ tot, uint32_t* __restrict__ err) {
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nr; t += gridDim.x * blockDim.x) {
        ChainNode c = node[rul[t]];
        uint64_t la = 0;
        uint32_t lc = 0, lm = c.pos;
        loc[c.pos] = SubPos{0, t, 0, lm, epoch, 0, 0};
        for (uint32_t step = 0; step < m && c.nx != INVALID; ++step) {
            if (c.nx >= n || node[c.nx].pos >= m) {  // a link out of the member set
                atomicExch(err, 1u);
                break;
            }
            const ChainNode d = node[c.nx];
            la += c.off;
            ++lc;
            if (d.rix != INVALID) break;
            lm = min(lm, d.pos);
            loc[d.pos] = SubPos{la, t, lc, lm, epoch, 0, 0};
            c = d;
        }
        tot[t] = SubTotal{la, lc, lm};
    }
}

// Members that no walk reached (cycles without a ruler).
__global__ void __launch_bounds__(256) unreached_kernel(uint32_t m, uint32_t epoch, const SubPos* __restrict__ loc,
                                                        uint8_t* __restrict__ flag, uint32_t* __restrict__ count) {
    uint32_t c = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        const bool u = loc[i].epoch != epoch;
        flag[i] = u;
        c += u;
    }
    block_tally<uint32_t>(c, count);
}

// On a cycle without a ruler, its member of smallest list index becomes
// one: each member walks the cycle (bounded by m steps) for the minimum.
__global__ void promote_kernel(const uint32_t* __restrict__ ids, uint32_t m, uint32_t n,
                               const uint8_t* __restrict__ unreached,
                               const uint32_t* __restrict__ nx, const uint32_t* __restrict__ pos_in_ids,
                               uint8_t* __restrict__ promote) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m || !unreached[i]) return;
    const uint32_t x = ids[i];
    uint32_t y = nx[x];
    bool smallest = true;
    for (uint32_t step = 0; step < m && y != x && y < n; ++step) {
        if (pos_in_ids[y] < i) {  // non-members hold INVALID
            smallest = false;
            break;
        }
        y = nx[y];
    }
    promote[i] = smallest;
}

// Ruler ranking state: the predecessor ruler owns the read before this
// ruler's first read.
__global__ void ruler_init_kernel(const uint32_t* __restrict__ rul, uint32_t nr, uint32_t m,
                                  const uint32_t* __restrict__ pv,
                                  const uint32_t* __restrict__ pos_in_ids, const SubPos* __restrict__ loc,
                                  const SubTotal* __restrict__ tot, RankState* __restrict__ st) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nr) return;
    const uint32_t p = pv[rul[t]];
    const uint32_t pi = p == INVALID ? INVALID : pos_in_ids[p];
    const uint32_t pr = pi < m ? loc[pi].owner : INVALID;
    RankState r;
    r.jump = pr;
    r.far = pr == INVALID ? t : pr;
    r.acc = pr == INVALID ? 0 : tot[pr].acc;
    r.cnt = pr == INVALID ? 0 : tot[pr].cnt;
    r.mn = tot[t].mn;
    if (pr != INVALID) r.mn = min(r.mn, tot[pr].mn);
    r.pad0 = r.pad1 = 0;
    st[t] = r;
}

// One jump for every ruler (grid-stride); *active counts the rulers whose
// pointer is still set afterwards.
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

// Member state = its ruler's + its place in the sublist.  jump stays set for
// members of a cycle.
__global__ void member_state_kernel(uint32_t m, const uint32_t* __restrict__ rul, const SubPos* __restrict__ loc,
                                    const RankState* __restrict__ rs, RankState* __restrict__ st) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const SubPos l = loc[i];
    const RankState r = rs[l.owner];
    RankState o;
    o.acc = r.acc + l.la;
    o.jump = r.jump;
    o.far = rul[r.far];
    o.cnt = r.cnt + l.lc;
    o.mn = min(r.mn, l.lm);
    o.pad0 = o.pad1 = 0;
    st[i] = o;
}

__global__ void cycle_flags_kernel(uint32_t m, const RankState* __restrict__ st, uint8_t* __restrict__ cyc) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) cyc[i] = st[i].jump != INVALID;
}

// Cycles are cut in parallel.  The reference walks each cycle from the
// successor h of its first listed read r (the read visited first) round to
// r, and cuts after the first read of largest offset met on the way.  Here:
// (1) a temporary cut between r and h makes each cycle a chain h .. r;
// (2) ranking that chain gives every read its walk position;
// (3) the largest (offset, -position) over the chain picks the cut read;
// (4) the temporary cut is undone and the real one made.

// (1) r = the cycle member whose list index is the cycle's minimum (mn on a
// cycle covers the whole cycle).
__global__ void cycle_open_kernel(const uint32_t* __restrict__ ids, uint32_t m, const RankState* __restrict__ st,
                                  const uint8_t* __restrict__ cyc, uint32_t* nx, uint32_t* pv,
                                  uint32_t* __restrict__ leader_of_head, uint32_t* __restrict__ err) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m || !cyc[i] || st[i].mn != i) return;
    const uint32_t x = ids[i];
    const uint32_t h = nx[x];
    if (h == INVALID || pv[h] != x) {
        atomicExch(err, 1u);
        return;
    }
    leader_of_head[h] = x;
    pv[h] = INVALID;
    nx[x] = INVALID;
}

// (3) per chain head: max of (offset << 32 | ~position)
__global__ void cycle_max_kernel(const uint32_t* __restrict__ ids, uint32_t m, const RankState* __restrict__ st,
                                 const uint8_t* __restrict__ cyc, const uint16_t* __restrict__ offset,
                                 unsigned long long* __restrict__ best) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m || !cyc[i]) return;
    const unsigned long long key = (unsigned long long)offset[ids[i]] << 32 | (0xFFFFFFFFu - st[i].cnt);
    atomicMax(&best[st[i].far], key);
}

// (4) the read that holds its chain's maximum restores the temporary cut and
// makes the real one after itself.
__global__ void cycle_cut_kernel(const uint32_t* __restrict__ ids, uint32_t m, const RankState* __restrict__ st,
                                 const uint8_t* __restrict__ cyc, const unsigned long long* __restrict__ best,
                                 const uint32_t* __restrict__ leader_of_head, uint32_t* nx, uint32_t* pv) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m || !cyc[i]) return;
    const uint32_t h = st[i].far;
    if ((0xFFFFFFFFu - uint32_t(best[h] & 0xFFFFFFFFull)) != st[i].cnt) return;
    const uint32_t r = leader_of_head[h];
    pv[h] = r;
    nx[r] = h;
    const uint32_t x = ids[i];
    const uint32_t nh = nx[x];
    nx[x] = INVALID;
    pv[nh] = INVALID;
}

// The cycle members as a list of their own (in list order).
__global__ void cycle_list_kernel(const uint32_t* __restrict__ ids, const uint32_t* __restrict__ cidx, uint32_t mc,
                                  uint32_t* __restrict__ cids, uint32_t* __restrict__ pos_in_cyc) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= mc) return;
    const uint32_t x = ids[cidx[t]];
    cids[t] = x;
    pos_in_cyc[x] = t;
}

// States of the cut cycles back into the full list (mn to a list index).
__global__ void cycle_merge_kernel(const uint32_t* __restrict__ cidx, uint32_t mc, const RankState* __restrict__ T,
                                   RankState* __restrict__ R) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= mc) return;
    RankState r = T[t];
    r.mn = cidx[r.mn];
    R[cidx[t]] = r;
}

// The chain's first list index, from its tail (whose mn covers the chain).
__global__ void chain_key_kernel(const uint32_t* __restrict__ ids, uint32_t m, const uint32_t* __restrict__ nx,
                                 const RankState* __restrict__ st, uint32_t* __restrict__ key) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m && nx[ids[i]] == INVALID) key[st[i].far] = st[i].mn;
}

__global__ void head_flags_kernel(const uint32_t* __restrict__ ids, uint32_t m, const uint32_t* __restrict__ pv,
                                  uint8_t* __restrict__ f) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) f[i] = pv[ids[i]] == INVALID;
}

__global__ void tail_sizes_kernel(const uint32_t* __restrict__ ids, uint32_t m, const uint32_t* __restrict__ nx,
                                  const RankState* __restrict__ st, int L, uint64_t* __restrict__ chain_bases,
                                  uint32_t* __restrict__ chain_members) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m || nx[ids[i]] != INVALID) return;
    chain_bases[st[i].far] = st[i].acc + uint64_t(L);
    chain_members[st[i].far] = st[i].cnt + 1;
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
    const RankState r = st[i];
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

// Scratch of one ranking, sized for m members of n reads.
struct RankScratch {
    ChainNode* node;
    SubPos* loc;
    uint8_t* flags;
    uint8_t* promote;
    uint32_t* rul;
    SubTotal* tot;
    RankState* A;
    RankState* B;
    uint32_t* counts;  // [0] rulers, [1] unreached, [2] active
    uint32_t epoch;    // walks so far (loc is zeroed once, so 0 is never current)
};

// Ranks every member: st[i] for list index i.  Returns the number of members
// on cycles (jump still set).
uint32_t rank_members(const uint32_t* ids, uint32_t m, uint32_t n, const uint32_t* nx, const uint32_t* pv,
                      const uint16_t* offset, const uint32_t* pos_in_ids, RankScratch& k, RankState* st,
                      Arena& a, cudaStream_t s) {
    const int g = grid_for(m, 256);
    const uint8_t* promote = nullptr;
    uint32_t nr = 0;
    SubStage sp_walk("assembly.walk");
    CURC_CHECK(cudaMemsetAsync(k.counts + 3, 0, 4, s));
    chain_nodes_kernel<<<resident_grid(chain_nodes_kernel, 256, n), 256, 0, s>>>(n, pos_in_ids, nx, offset, k.node);
    CURC_LAUNCH_CHECK();
    for (int attempt = 0; attempt < 2; ++attempt) {
        const uint32_t epoch = ++k.epoch;
        ruler_flags_kernel<<<g, 256, 0, s>>>(ids, m, pv, promote, k.flags);
        CURC_LAUNCH_CHECK();
        select_flagged(ids, k.flags, k.rul, m, k.counts, a, s);
        if (attempt) {  // clear the ruler marks of the first attempt
            chain_nodes_kernel<<<resident_grid(chain_nodes_kernel, 256, n), 256, 0, s>>>(n, pos_in_ids, nx, offset,
                                                                                          k.node);
            CURC_LAUNCH_CHECK();
        }
        CURC_CHECK(cudaMemsetAsync(k.counts + 1, 0, 4, s));
        nr = read_scalar(k.counts, s);
        ruler_index_kernel<<<grid_for(nr, 256), 256, 0, s>>>(k.rul, nr, k.node);
        CURC_LAUNCH_CHECK();
        ruler_walk_kernel<<<resident_grid(ruler_walk_kernel, 256, nr), 256, 0, s>>>(k.rul, nr, m, n, epoch, k.node,
                                                                                    k.loc, k.tot, k.counts + 3);
        CURC_LAUNCH_CHECK();
        unreached_kernel<<<resident_grid(unreached_kernel, 256, m), 256, 0, s>>>(m, epoch, k.loc, k.flags,
                                                                                  k.counts + 1);
        CURC_LAUNCH_CHECK();
        uint32_t hc[4];
        read_small(hc, k.counts, 16, s);
        if (hc[3]) throw std::runtime_error("assemble: a chain link leaves the member set");
        if (hc[1] == 0) break;
        if (attempt == 1) throw std::runtime_error("assemble: reads left unranked after promoting cycle rulers");
        CURC_CHECK(cudaMemsetAsync(k.promote, 0, m, s));
        promote_kernel<<<g, 256, 0, s>>>(ids, m, n, k.flags, nx, pos_in_ids, k.promote);
        CURC_LAUNCH_CHECK();
        promote = k.promote;
    }
    sp_walk.stop();
    SubStage sp_jump("assembly.jump");
    ruler_init_kernel<<<grid_for(nr, 256), 256, 0, s>>>(k.rul, nr, m, pv, pos_in_ids, k.loc, k.tot, k.A);
    CURC_LAUNCH_CHECK();
    RankState* A = k.A;
    RankState* B = k.B;
    uint32_t left = 0;
    // the count of pointers left is read every few rounds (a round on
    // converged states changes nothing)
    const int R = rounds_for(nr);
    const int gs = resident_grid(rank_step_kernel, 512, nr);
    for (int t = 0; t < R; ++t) {
        CURC_CHECK(cudaMemsetAsync(k.counts + 2, 0, 4, s));
        rank_step_kernel<<<gs, 512, 0, s>>>(nr, A, B, k.counts + 2);
        CURC_LAUNCH_CHECK();
        std::swap(A, B);
        if (t % 4 != 3 && t + 1 < R) continue;
        left = read_scalar(k.counts + 2, s);
        if (left == 0) break;
    }
    member_state_kernel<<<g, 256, 0, s>>>(m, k.rul, k.loc, A, st);
    CURC_LAUNCH_CHECK();
    return left;
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
    SubStage sp_rank("assembly.ranking");
    RankScratch k;
    k.node = a.alloc<ChainNode>(n);
    k.loc = a.alloc<SubPos>(m);
    CURC_CHECK(cudaMemsetAsync(k.loc, 0, size_t(m) * sizeof(SubPos), s));
    k.epoch = 0;
    k.flags = a.alloc<uint8_t>(m);
    k.promote = a.alloc<uint8_t>(m);
    k.rul = a.alloc<uint32_t>(m);
    k.tot = a.alloc<SubTotal>(m);
    k.A = a.alloc<RankState>(m);
    k.B = a.alloc<RankState>(m);
    k.counts = a.alloc<uint32_t>(4);
    RankState* R = a.alloc<RankState>(m);
    uint32_t left = rank_members(ids, m, n_total, nx, pv, offset, pos_in_ids, k, R, a, s);
    if (left) {
        // Cycles: cut each in parallel.  Only their members are ranked again
        // (a cut cycle is a chain of exactly its members), as a list of its
        // own in list order, and their states are then written back.
        uint8_t* cyc = a.alloc<uint8_t>(m);
        cycle_flags_kernel<<<g, 256, 0, s>>>(m, R, cyc);
        CURC_LAUNCH_CHECK();
        uint32_t* leader_of_head = a.alloc<uint32_t>(n);
        unsigned long long* best = a.alloc<unsigned long long>(n);
        CURC_CHECK(cudaMemsetAsync(best, 0, n * sizeof(unsigned long long), s));
        CURC_CHECK(cudaMemsetAsync(k.counts + 3, 0, 4, s));
        cycle_open_kernel<<<g, 256, 0, s>>>(ids, m, R, cyc, nx, pv, leader_of_head, k.counts + 3);
        CURC_LAUNCH_CHECK();
        uint32_t* cidx = a.alloc<uint32_t>(m);
        select_indices(cyc, cidx, m, k.counts + 2, a, s);
        uint32_t hc[2];
        read_small(hc, k.counts + 2, 8, s);
        if (hc[1]) throw std::runtime_error("assemble: broken cycle");
        const uint32_t mc = hc[0];
        const int gc = grid_for(mc, 256);
        uint32_t* cids = a.alloc<uint32_t>(mc);
        uint32_t* pos_in_cyc = a.alloc<uint32_t>(n);
        fill<uint32_t>(pos_in_cyc, INVALID, n, s);
        cycle_list_kernel<<<gc, 256, 0, s>>>(ids, cidx, mc, cids, pos_in_cyc);
        CURC_LAUNCH_CHECK();
        uint8_t* all = a.alloc<uint8_t>(mc);
        CURC_CHECK(cudaMemsetAsync(all, 1, mc, s));
        RankScratch kc;
        kc.node = k.node;
        kc.loc = a.alloc<SubPos>(mc);
        CURC_CHECK(cudaMemsetAsync(kc.loc, 0, size_t(mc) * sizeof(SubPos), s));
        kc.epoch = 0;
        kc.flags = a.alloc<uint8_t>(mc);
        kc.promote = a.alloc<uint8_t>(mc);
        kc.rul = a.alloc<uint32_t>(mc);
        kc.tot = a.alloc<SubTotal>(mc);
        kc.A = a.alloc<RankState>(mc);
        kc.B = a.alloc<RankState>(mc);
        kc.counts = a.alloc<uint32_t>(4);
        RankState* T = a.alloc<RankState>(mc);
        if (rank_members(cids, mc, n_total, nx, pv, offset, pos_in_cyc, kc, T, a, s))
            throw std::runtime_error("assemble: cycle still closed after its temporary cut");
        cycle_max_kernel<<<gc, 256, 0, s>>>(cids, mc, T, all, offset, best);
        CURC_LAUNCH_CHECK();
        cycle_cut_kernel<<<gc, 256, 0, s>>>(cids, mc, T, all, best, leader_of_head, nx, pv);
        CURC_LAUNCH_CHECK();
        if (rank_members(cids, mc, n_total, nx, pv, offset, pos_in_cyc, kc, T, a, s))
            throw std::runtime_error("assemble: unresolved chain links after cutting cycles");
        cycle_merge_kernel<<<gc, 256, 0, s>>>(cidx, mc, T, R);
        CURC_LAUNCH_CHECK();
    }
    sp_rank.stop();
    SubStage sp_place("assembly.order_place");
    // chain order: first member in list order
    uint32_t* key = a.alloc<uint32_t>(n);
    chain_key_kernel<<<g, 256, 0, s>>>(ids, m, nx, R, key);
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
