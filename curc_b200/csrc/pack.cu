// a1: 2-bit read packing and N-read separation.
//
// Reference: encode() compress.cu:2151-2180 (one thread per read, strided
// byte loads) and the N test of the host parser, preprocess.cpp:147-193.
//
// B200 design: a persistent grid walks tiles of 64 reads.  Each tile is
// 64*L contiguous bytes, moved into shared memory by a 1D TMA bulk copy
// (cp.async.bulk + mbarrier) two tiles ahead of the compute, so HBM reads
// are full-line and overlap the packing.  Each thread then packs one output
// word (32 bases) from shared memory; packed words of a tile are contiguous
// in HBM, so stores coalesce.  Bytes per read: L in, 8*W + 1 out.
#include "stages.cuh"

namespace curc {

namespace {
constexpr int PACK_READS = 64;
constexpr int PACK_THREADS = 256;
constexpr uint32_t WAIT_LIMIT = 1u << 26;

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
// eight bits, first base in the top two: bits 1-3 of the letters give
// A/a 0, C/c 1, G/g 2, T/t 3 as ((c >> 1) ^ (c >> 2)) & 3, and one multiply
// gathers the four 2-bit codes into the top byte.
__device__ __forceinline__ uint32_t pack4(uint32_t x) {
    const uint32_t t = ((x >> 1) ^ (x >> 2)) & 0x03030303u;
    return (t * 0x40100401u) >> 24;
}

// The four bytes are all uppercase A, C, G or T (the common case, where
// pack4 is exact and no N is present): rebuild them from their codes.
__device__ __forceinline__ bool plain4(uint32_t x) {
    const uint32_t t = ((x >> 1) ^ (x >> 2)) & 0x03030303u;
    const uint32_t sel = (t & 3u) | ((t >> 4) & 0x30u) | ((t >> 8) & 0x300u) | ((t >> 12) & 0x3000u);
    return __byte_perm(0x54474341u, 0u, sel) == x;
}

__global__ void __launch_bounds__(PACK_THREADS) pack_kernel(const uint8_t* __restrict__ seq, uint64_t n, int L, int W,
                                                             uint32_t tile_bytes, bool use_tma,
                                                             uint64_t* __restrict__ packed, uint8_t* __restrict__ has_n,
                                                             uint32_t* __restrict__ err) {
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ uint8_t nflag[PACK_READS];
    const uint64_t tiles = div_up(n, PACK_READS);
    // a word's loads may run 36 bytes past its row: keep them in the buffer
    const uint32_t stride_bytes = (tile_bytes + 64u + 127u) & ~127u;
    auto full = [&](uint64_t t) { return (t + 1) * PACK_READS <= n; };
    auto issue = [&](uint64_t t, int stage) {
        mbar_expect_tx(&bar[stage], tile_bytes);
        bulk_g2s(smem + stage * stride_bytes, seq + t * uint64_t(PACK_READS) * L, tile_bytes, &bar[stage]);
    };
    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    uint64_t t = blockIdx.x;
    if (use_tma && threadIdx.x == 0 && t < tiles && full(t)) issue(t, 0);
    bool pending[2] = {use_tma && t < tiles && full(t), false};
    for (uint32_t it = 0; t < tiles; t += gridDim.x, ++it) {
        const int stage = it & 1;
        const uint64_t nt = t + gridDim.x;
        if (use_tma && nt < tiles && full(nt)) {
            if (threadIdx.x == 0) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                issue(nt, stage ^ 1);
            }
            pending[stage ^ 1] = true;
        }
        uint8_t* buf = smem + stage * stride_bytes;
        const uint64_t rem = n - t * PACK_READS;
        const uint32_t nr = rem < uint64_t(PACK_READS) ? uint32_t(rem) : uint32_t(PACK_READS);
        if (pending[stage]) {
            uint32_t spins = 0;
            while (!mbar_try_wait(&bar[stage], (it >> 1) & 1)) {
                if (++spins > WAIT_LIMIT) {  // never expected: report and stop cleanly
                    if (threadIdx.x == 0) atomicExch(err, 1u);
                    break;
                }
            }
            pending[stage] = false;
        } else {
            const uint8_t* src = seq + t * uint64_t(PACK_READS) * L;
            for (uint32_t b = threadIdx.x; b < nr * uint32_t(L); b += PACK_THREADS) buf[b] = src[b];
        }
        if (threadIdx.x < PACK_READS) nflag[threadIdx.x] = 0;
        __syncthreads();
        for (uint32_t item = threadIdx.x; item < nr * uint32_t(W); item += PACK_THREADS) {
            const uint32_t r = item / W, w = item - r * W;
            const uint32_t a = r * uint32_t(L) + w * 32;
            const int nb = min(32, L - int(w) * 32);
            // eight 4-byte groups from aligned shared-memory words; bytes past
            // the read's end are replaced by 'A' (code 0, the zero padding)
            const uint32_t* b32 = reinterpret_cast<const uint32_t*>(buf + (a & ~3u));
            const uint32_t sh = (a & 3u) * 8u;
            uint32_t lo = b32[0];
            uint64_t v = 0;
            bool plain = true;
#pragma unroll
            for (int g = 0; g < 8; ++g) {
                const uint32_t hi = b32[g + 1];
                uint32_t x = __funnelshift_r(lo, hi, sh);
                lo = hi;
                const int vb = nb - 4 * g;
                if (vb < 4) {
                    const uint32_t keep = vb <= 0 ? 0u : (1u << (8 * vb)) - 1u;
                    x = (x & keep) | (0x41414141u & ~keep);
                }
                v = (v << 8) | pack4(x);
                plain &= plain4(x);
            }
            if (!plain) {  // N, lower case or other letters: byte by byte
                const uint8_t* sb = buf + a;
                bool hn = false;
                v = 0;
                for (int j = 0; j < nb; ++j) {
                    const uint8_t c = sb[j];
                    hn |= (c == 'N');
                    v = (v << 2) | uint64_t(ascii_code(c));
                }
                v <<= 2 * (32 - nb);
                if (hn) nflag[r] = 1;
            }
            packed[(t * PACK_READS + r) * W + w] = v;
        }
        __syncthreads();
        if (threadIdx.x < nr) has_n[t * PACK_READS + threadIdx.x] = nflag[threadIdx.x];
        __syncthreads();
    }
    // drain a prefetch that was issued but not consumed (cannot happen: a
    // prefetch is only issued for a tile this block will process)
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
    const uint32_t tile_bytes = uint32_t(PACK_READS) * uint32_t(L);
    const bool aligned = (reinterpret_cast<uintptr_t>(seq) & 15u) == 0;
    const size_t smem = 2 * ((tile_bytes + 64u + 127u) & ~127u);
    static bool attr_set = false;
    if (!attr_set) {
        CURC_CHECK(cudaFuncSetAttribute(pack_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        2 * (64 * 512 + 64 + 128)));
        attr_set = true;
    }
    const uint64_t tiles = div_up(n, PACK_READS);
    const int grid = int(std::min<uint64_t>(tiles, uint64_t(SM_COUNT_B200) * 8));
    pack_kernel<<<grid, PACK_THREADS, smem, s>>>(seq, n, L, W, tile_bytes, aligned, packed, has_n, err);
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
