// a1: 2-bit read packing and N-read separation.
//
// Reference: encode() compress.cu:2151-2180 (one thread per read, strided
// byte loads) and the N test of the host parser, preprocess.cpp:147-193.
//
// B200 design: a persistent grid walks tiles of 64 reads.  Each tile is
// 64*L contiguous bytes, moved into shared memory by a 1D TMA bulk copy
// (cp.async.bulk + mbarrier) one tile ahead of the compute (two stages),
// so HBM reads are full-line and the copies overlap the packing; with two
// stages a block's shared memory is small enough for 9 blocks per SM at
// 150 bp, and the packing itself (a few instructions per byte) is what
// more resident warps hide.  The block then works in two
// conflict-free passes: every thread turns 16-byte groups of the tile into
// 32 bits of codes (one 16-byte shared-memory load each), giving the tile's
// bases as one contiguous 2-bit string, and then every thread cuts one
// output word (32 bases) per read of its column out of that string.  A
// block has 32*W threads, so both passes keep every thread busy; packed
// words of a tile are contiguous in HBM, so stores coalesce.  Bytes per
// read: L in, 8*W + 1 out.
#include <mutex>
#include <stdexcept>

#include "stages.cuh"

namespace curc {

namespace {
constexpr int PACK_READS = 64;
constexpr int PACK_STAGES = 2;  // tiles in flight per block: PACK_STAGES - 1 copies ahead of the compute
constexpr uint32_t WAIT_LIMIT = 1u << 26;
constexpr int MAX_DEVICES = 64;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// Four ASCII bases (a little-endian word, first base in the low byte) to
// their 2-bit codes, one per byte: bits 1-3 of the letters give A/a 0,
// C/c 1, G/g 2, T/t 3 as ((c >> 1) ^ (c >> 2)) & 3.
__device__ __forceinline__ uint32_t codes4(uint32_t x) { return ((x >> 1) ^ (x >> 2)) & 0x03030303u; }

// The codes as eight bits, first base in the top two, in the top byte of
// the product (one multiply gathers them; no partial product carries into
// that byte).
__device__ __forceinline__ uint32_t gather4(uint32_t t) { return t * 0x40100401u; }

// The letters that four codes stand for, in lower case ("acgt"[t_i] in
// byte i).  u's byte 0 holds t0 | t1 << 4 and its byte 2 t2 | t3 << 4, so
// one permute makes them the lookup's selector.  The four input bytes are
// all A, C, G or T in either case exactly when this equals (x | 0x20202020):
// setting bit 5 merges only a letter with its other case.
__device__ __forceinline__ uint32_t letters4(uint32_t t) {
    const uint32_t u = t | (t >> 4);
    return __byte_perm(0x74676361u, 0u, __byte_perm(u, 0u, 0x4420u));
}

// Shared memory of one stage: the tile's bytes (a multiple of 128), then
// its codes (4*L words of 16 bases, and 4 zero words after them).
__host__ __device__ inline uint32_t pack_tile_stride(int L) { return (uint32_t(PACK_READS) * L + 127u) & ~127u; }
__host__ __device__ inline uint32_t pack_code_words(int L) { return 4u * uint32_t(L) + 4u; }
inline size_t pack_smem_bytes(int L) {
    return PACK_STAGES * (size_t(pack_tile_stride(L)) + 4 * size_t(pack_code_words(L)));
}

__global__ void __launch_bounds__(512) pack_kernel(const uint8_t* __restrict__ seq, uint64_t n, int L, int W,
                                                   bool use_tma, uint64_t* __restrict__ packed,
                                                   uint8_t* __restrict__ has_n, uint32_t* __restrict__ err) {
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t bar[PACK_STAGES];
    __shared__ uint8_t nflag[PACK_STAGES][PACK_READS];
    const uint32_t tile_bytes = uint32_t(PACK_READS) * uint32_t(L);
    const uint32_t groups = tile_bytes / 16;  // 4*L
    const uint32_t stride = pack_tile_stride(L);
    uint32_t* codes_base = reinterpret_cast<uint32_t*>(smem + PACK_STAGES * stride);
    const uint32_t cw = pack_code_words(L);
    const uint64_t tiles = div_up(n, PACK_READS);
    auto full = [&](uint64_t t) { return (t + 1) * PACK_READS <= n; };
    auto issue = [&](uint64_t t, int stage) {
        mbar_expect_tx(&bar[stage], tile_bytes);
        bulk_g2s(smem + stage * stride, seq + t * uint64_t(PACK_READS) * L, tile_bytes, &bar[stage]);
    };
    if (threadIdx.x == 0) {
        for (int st = 0; st < PACK_STAGES; ++st) mbar_init(&bar[st], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (uint32_t i = threadIdx.x; i < PACK_STAGES * PACK_READS; i += blockDim.x)
        nflag[i / PACK_READS][i % PACK_READS] = 0;
    if (threadIdx.x < 4 * PACK_STAGES) codes_base[(threadIdx.x / 4) * cw + groups + threadIdx.x % 4] = 0;
    __syncthreads();
    // this thread's output column: word w0 of reads r0, r0 + 32, ...
    const uint32_t r0 = threadIdx.x / uint32_t(W), w0 = threadIdx.x - r0 * uint32_t(W);
    const int nb = min(32, L - int(w0) * 32);
    const uint64_t tail_mask = nb < 32 ? ~0ull << (64 - 2 * nb) : ~0ull;
    uint64_t t = blockIdx.x;
    uint32_t pending = 0;  // bit s: a copy into stage s is in flight
    for (int j = 0; j + 1 < PACK_STAGES; ++j) {
        const uint64_t tj = t + uint64_t(j) * gridDim.x;
        if (use_tma && tj < tiles && full(tj)) {
            if (threadIdx.x == 0) issue(tj, j);
            pending |= 1u << j;
        }
    }
    uint32_t it = 0;
    for (; t < tiles; t += gridDim.x, ++it) {
        const int stage = int(it % PACK_STAGES);
        const int ahead = int((it + PACK_STAGES - 1) % PACK_STAGES);  // the stage iteration it-1 used
        const uint64_t nt = t + uint64_t(PACK_STAGES - 1) * gridDim.x;
        if (use_tma && nt < tiles && full(nt)) {
            if (threadIdx.x == 0) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                issue(nt, ahead);
            }
            pending |= 1u << ahead;
        }
        uint8_t* buf = smem + stage * stride;
        uint32_t* codes = codes_base + stage * cw;
        uint8_t* nf = nflag[stage];
        const uint64_t rem = n - t * PACK_READS;
        const uint32_t nr = rem < uint64_t(PACK_READS) ? uint32_t(rem) : uint32_t(PACK_READS);
        if (pending >> stage & 1u) {
            uint32_t spins = 0;
            bool late = false;
            while (!mbar_try_wait(&bar[stage], (it / PACK_STAGES) & 1)) {
                if (++spins > WAIT_LIMIT) {  // never expected
                    late = true;
                    break;
                }
            }
            pending &= ~(1u << stage);
            if (__syncthreads_or(late)) {
                // report, write nothing of this tile, and leave only once the
                // other stage's copy (if one is in flight) has also landed or
                // had the same bounded wait, so that, as far as waiting can
                // tell, no bulk copy still targets this block's shared memory
                if (threadIdx.x == 0) {
                    atomicExch(err, 1u);
                    for (int d = 1; d < PACK_STAGES; ++d) {
                        const int other = int((it + d) % PACK_STAGES);  // holds the copy for iteration it + d
                        if (pending >> other & 1u) {
                            const uint32_t par = ((it + d) / PACK_STAGES) & 1;
                            for (uint32_t w = 0; w < WAIT_LIMIT && !mbar_try_wait(&bar[other], par); ++w) {
                            }
                        }
                    }
                }
                __syncthreads();
                return;
            }
        } else {
            // the last, partial tile: plain loads, the rest of the tile 'A'
            const uint8_t* src = seq + t * uint64_t(PACK_READS) * L;
            const uint32_t have = nr * uint32_t(L);
            for (uint32_t b = threadIdx.x; b < tile_bytes; b += blockDim.x) buf[b] = b < have ? src[b] : 'A';
        }
        __syncthreads();
        // pass 1: 16 bytes -> 32 bits of codes, first base in the top bits
        for (uint32_t g = threadIdx.x; g < groups; g += blockDim.x) {
            const uint4 x = reinterpret_cast<const uint4*>(buf)[g];
            const uint32_t t0 = codes4(x.x), t1 = codes4(x.y), t2 = codes4(x.z), t3 = codes4(x.w);
            // the top bytes of the four products: byte 3 from the first word
            uint32_t c = __byte_perm(__byte_perm(gather4(t3), gather4(t2), 0x0073u),
                                     __byte_perm(gather4(t1), gather4(t0), 0x0073u), 0x5410u);
            const uint32_t d = (letters4(t0) ^ (x.x | 0x20202020u)) | (letters4(t1) ^ (x.y | 0x20202020u)) |
                               (letters4(t2) ^ (x.z | 0x20202020u)) | (letters4(t3) ^ (x.w | 0x20202020u));
            if (d != 0) {
                // N, other letters: byte by byte
                c = 0;
                for (uint32_t j = 0; j < 16; ++j) {
                    const uint8_t ch = buf[16 * g + j];
                    c = (c << 2) | uint32_t(ascii_code(ch));
                    if (ch == 'N') nf[(16 * g + j) / uint32_t(L)] = 1;
                }
            }
            codes[g] = c;
        }
        __syncthreads();
        // pass 2: the 32 bases of word w0 of each read, from the code string
        for (uint32_t r = r0; r < nr; r += 32) {
            const uint32_t o = r * uint32_t(L) + 32u * w0;
            const uint32_t k = o >> 4, sh = (o & 15u) * 2u;
            uint64_t v = (uint64_t(codes[k]) << 32) | codes[k + 1];
            if (sh) v = (v << sh) | (codes[k + 2] >> (32u - sh));
            packed[(t * PACK_READS + r) * W + w0] = v & tail_mask;
        }
        for (uint32_t i = threadIdx.x; i < nr; i += blockDim.x) {
            has_n[t * PACK_READS + i] = nf[i];
            nf[i] = 0;
        }
    }
}

__global__ void invert_flags_kernel(const uint8_t* __restrict__ in, uint8_t* __restrict__ out, uint64_t n) {
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
        out[i] = in[i] ? 0 : 1;
}

__global__ void gather_reads_ascii_kernel(const uint8_t* __restrict__ seq, const uint32_t* __restrict__ ids,
                                          uint32_t m, int L, uint8_t* __restrict__ out) {
    // one warp per read
    const uint32_t warp = (uint32_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= m) return;
    const uint8_t* s = seq + uint64_t(ids[warp]) * L;
    uint8_t* d = out + uint64_t(warp) * L;
    for (int j = lane; j < L; j += 32) d[j] = s[j];
}
}  // namespace

void pack_reads(const uint8_t* seq, uint64_t n, int L, uint64_t* packed, uint8_t* has_n, uint32_t* err,
                cudaStream_t s) {
    if (n == 0) return;
    const int W = (L + 31) / 32;
    const bool aligned = (reinterpret_cast<uintptr_t>(seq) & 15u) == 0;
    const size_t smem = pack_smem_bytes(L);
    // the dynamic shared-memory limit is a per-device attribute: raise it
    // once on every device this process packs on
    static std::mutex mu;
    static bool attr_set[MAX_DEVICES] = {};
    int dev = 0;
    CURC_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= MAX_DEVICES) throw std::runtime_error("device ordinal out of range");
    {
        std::lock_guard<std::mutex> g(mu);
        if (!attr_set[dev]) {
            CURC_CHECK(cudaFuncSetAttribute(pack_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            int(pack_smem_bytes(512))));
            attr_set[dev] = true;
        }
    }
    const int threads = 32 * W;
    int per_sm = 0;
    CURC_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pack_kernel, threads, smem));
    const uint64_t tiles = div_up(n, PACK_READS);
    const int grid = int(std::min<uint64_t>(tiles, uint64_t(SM_COUNT_B200) * uint64_t(std::max(1, per_sm))));
    pack_kernel<<<grid, threads, smem, s>>>(seq, n, L, W, aligned, packed, has_n, err);
    CURC_LAUNCH_CHECK();
}

void split_n_reads(const uint8_t* has_n, uint64_t n, uint32_t* reads_id, uint32_t* n_reads_id, uint32_t* counts,
                   Arena& a, cudaStream_t s) {
    // preprocess.cpp:147-193: ids of reads without N ascending, ids of reads
    // with N ascending.
    auto m = a.mark();
    uint8_t* inv = a.alloc<uint8_t>(n ? n : 1);
    if (n) {
        invert_flags_kernel<<<grid_for(n, 256, 4), 256, 0, s>>>(has_n, inv, n);
        CURC_LAUNCH_CHECK();
    }
    select_indices(inv, reads_id, n, counts + 0, a, s);
    select_indices(has_n, n_reads_id, n, counts + 1, a, s);
    a.release(m);
}

void gather_ascii_rows(const uint8_t* seq, const uint32_t* ids, uint32_t m, int L, uint8_t* out, cudaStream_t s) {
    if (!m) return;
    gather_reads_ascii_kernel<<<grid_for(uint64_t(m) * 32, 256), 256, 0, s>>>(seq, ids, m, L, out);
    CURC_LAUNCH_CHECK();
}

}  // namespace curc
