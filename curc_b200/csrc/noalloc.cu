// curc_pack_split_noalloc: 2-bit packing plus N-read separation without any
// device allocation.
//
// Who needs it: a host application that owns all device memory itself (it
// reserves HBM up front through its own pool and forbids stray cudaMalloc
// calls, e.g. to stay inside a fixed memory budget next to other tenants),
// or a caller that cannot afford the implicit device synchronisation a
// cudaMalloc / cudaFree may perform in the middle of its stream work.  The
// regular entry points take their scratch from a context arena, which grows
// with cudaMalloc; this one takes it from a fixed array compiled into the
// library.
//
// Scratch: `g_split_scratch`, a file-scope static __device__ array of
// 2 * 65536 + 64 words (about 512 KB), holding the per-tile counts of the
// two compactions and the error word.  Every GPU that loads the library
// holds it until the process exits.  It bounds a call to 2^27 reads (65536
// tiles of 2048); larger calls are rejected.  All calls share the array and
// it keeps the last call's contents: every word a call reads is written by
// that call first (the error word is cleared on the stream), so calls that
// are stream-ordered are independent, but calls that overlap on the GPU
// (different streams, or different host threads, without ordering) race on
// it and must not be issued.
//
// Host code cannot use the array's name as a device address.  The first
// call on a device, with that device current, looks the address up with
// cudaGetSymbolAddress and caches it; that first call therefore also loads
// the module, and should come before any stream capture.  The cached
// address belongs to the device's primary context: after cudaDeviceReset
// (or any teardown of that context) it is stale, so a process that resets a
// device must not call this entry point on it again.
#include <mutex>
#include <string>

#include "../../include/curc_b200.h"
#include "stages.cuh"

namespace curc {

namespace {

constexpr uint64_t SPLIT_MAX_READS = 1ull << 27;
constexpr uint32_t SPLIT_TILE = 2048;
constexpr uint32_t SPLIT_TILES = uint32_t(SPLIT_MAX_READS / SPLIT_TILE);  // 65536
constexpr uint32_t SPLIT_THREADS = 256, SPLIT_ITEMS = SPLIT_TILE / SPLIT_THREADS;
constexpr uint32_t SCRATCH_WORDS = 2 * SPLIT_TILES + 64;
constexpr uint32_t ERR_WORD = 2 * SPLIT_TILES;

static __device__ __align__(256) uint32_t g_split_scratch[SCRATCH_WORDS];

constexpr int MAX_DEVICES = 64;
std::mutex g_addr_mu;
uint32_t* g_addr[MAX_DEVICES] = {nullptr};

__device__ uint32_t block_excl_sum(uint32_t v, uint32_t* total) {
    __shared__ uint32_t ws[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) ws[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < nw ? ws[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < nw) ws[lane] = w;
    }
    __syncthreads();
    const uint32_t pre = warp ? ws[warp - 1] : 0;
    *total = ws[nw - 1];
    __syncthreads();
    return pre + x - v;
}

// Per tile: number of reads without N and with N.
__global__ void __launch_bounds__(SPLIT_THREADS) split_count_kernel(const uint8_t* __restrict__ has_n, uint64_t n,
                                                                    uint32_t* __restrict__ scratch) {
    const uint64_t base = uint64_t(blockIdx.x) * SPLIT_TILE;
    uint32_t c = 0;
    for (uint32_t i = threadIdx.x; i < SPLIT_TILE; i += SPLIT_THREADS) {
        const uint64_t r = base + i;
        if (r < n) c += has_n[r] != 0;
    }
    uint32_t nn;
    block_excl_sum(c, &nn);
    if (threadIdx.x == 0) {
        const uint64_t rest = n - base;
        const uint32_t in_tile = rest < SPLIT_TILE ? uint32_t(rest) : SPLIT_TILE;
        scratch[blockIdx.x] = in_tile - nn;
        scratch[SPLIT_TILES + blockIdx.x] = nn;
    }
}

// Exclusive scan of the tile counts of one list (blockIdx.x = list), in
// place; the list's total goes to counts[list].
__global__ void __launch_bounds__(1024) split_scan_kernel(uint32_t tiles, uint32_t* __restrict__ scratch,
                                                          uint32_t* __restrict__ counts) {
    uint32_t* c = scratch + blockIdx.x * SPLIT_TILES;
    const uint32_t per = (tiles + blockDim.x - 1) / blockDim.x;
    const uint32_t lo = threadIdx.x * per, hi = min(tiles, lo + per);
    uint32_t s = 0;
    for (uint32_t t = lo; t < hi; ++t) s += c[t];
    uint32_t total;
    uint32_t run = block_excl_sum(s, &total);
    for (uint32_t t = lo; t < hi; ++t) {
        const uint32_t v = c[t];
        c[t] = run;
        run += v;
    }
    if (threadIdx.x == 0) counts[blockIdx.x] = total;
}

// Stable scatter of the read ids of both lists.
__global__ void __launch_bounds__(SPLIT_THREADS) split_scatter_kernel(const uint8_t* __restrict__ has_n, uint64_t n,
                                                                      const uint32_t* __restrict__ scratch,
                                                                      uint32_t* __restrict__ reads_id,
                                                                      uint32_t* __restrict__ n_reads_id) {
    const uint64_t base = uint64_t(blockIdx.x) * SPLIT_TILE + uint64_t(threadIdx.x) * SPLIT_ITEMS;
    uint8_t f[SPLIT_ITEMS];
    uint32_t cn = 0;
#pragma unroll
    for (uint32_t i = 0; i < SPLIT_ITEMS; ++i) {
        const uint64_t r = base + i;
        f[i] = r < n ? (has_n[r] != 0 ? 1 : 2) : 0;
        cn += f[i] == 1;
    }
    const uint32_t valid = base < n ? (n - base < SPLIT_ITEMS ? uint32_t(n - base) : SPLIT_ITEMS) : 0;
    uint32_t tn, tp;
    uint32_t pn = block_excl_sum(cn, &tn) + scratch[SPLIT_TILES + blockIdx.x];
    uint32_t pp = block_excl_sum(valid - cn, &tp) + scratch[blockIdx.x];
#pragma unroll
    for (uint32_t i = 0; i < SPLIT_ITEMS; ++i) {
        if (f[i] == 1) n_reads_id[pn++] = uint32_t(base + i);
        else if (f[i] == 2) reads_id[pp++] = uint32_t(base + i);
    }
}

int fail(int code, const std::string& msg) {
    ctxless_error() = msg;  // read back with curc_last_error(NULL)
    return code;
}

}  // namespace

}  // namespace curc

extern "C" int curc_pack_split_noalloc(int device, const char* seqs_dev, uint64_t n, uint16_t read_len,
                                       uint64_t* packed_dev, uint8_t* has_n_dev, uint32_t* reads_id_dev,
                                       uint32_t* n_reads_id_dev, uint32_t* counts_dev, void* stream) {
    using namespace curc;
    if (n > SPLIT_MAX_READS)
        return fail(CURC_ERR_ARG, "curc_pack_split_noalloc: " + std::to_string(n) +
                                      " reads exceed the fixed scratch limit of 134217728 (2^27) reads per call");
    if (read_len < 1 || read_len > 512) return fail(CURC_ERR_ARG, "curc_pack_split_noalloc: read length must be in [1, 512]");
    if (device < 0 || device >= MAX_DEVICES) return fail(CURC_ERR_ARG, "curc_pack_split_noalloc: bad device index");
    if (n && (!seqs_dev || !packed_dev || !has_n_dev || !reads_id_dev || !n_reads_id_dev))
        return fail(CURC_ERR_ARG, "curc_pack_split_noalloc: null buffer");
    if (!counts_dev) return fail(CURC_ERR_ARG, "curc_pack_split_noalloc: null counts buffer");
    try {
        CURC_CHECK(cudaSetDevice(device));
        uint32_t* scratch;
        {
            std::lock_guard<std::mutex> g(g_addr_mu);
            if (!g_addr[device]) {
                void* p = nullptr;
                cudaError_t e = cudaGetSymbolAddress(&p, g_split_scratch);
                if (e != cudaSuccess)
                    return fail(CURC_ERR_CUDA, std::string("curc_pack_split_noalloc: cudaGetSymbolAddress: ") +
                                                   cudaGetErrorString(e));
                g_addr[device] = static_cast<uint32_t*>(p);
            }
            scratch = g_addr[device];
        }
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        CURC_CHECK(cudaMemsetAsync(counts_dev, 0, 2 * sizeof(uint32_t), s));
        if (n == 0) return CURC_OK;
        uint32_t* err = scratch + ERR_WORD;
        CURC_CHECK(cudaMemsetAsync(err, 0, sizeof(uint32_t), s));
        pack_reads(reinterpret_cast<const uint8_t*>(seqs_dev), n, read_len, packed_dev, has_n_dev, err, s);
        const uint32_t tiles = uint32_t(div_up(n, SPLIT_TILE));
        split_count_kernel<<<tiles, SPLIT_THREADS, 0, s>>>(has_n_dev, n, scratch);
        CURC_LAUNCH_CHECK();
        split_scan_kernel<<<2, 1024, 0, s>>>(tiles, scratch, counts_dev);
        CURC_LAUNCH_CHECK();
        split_scatter_kernel<<<tiles, SPLIT_THREADS, 0, s>>>(has_n_dev, n, scratch, reads_id_dev, n_reads_id_dev);
        CURC_LAUNCH_CHECK();
        uint32_t herr = 0;
        CURC_CHECK(cudaMemcpyAsync(&herr, err, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        CURC_CHECK(cudaStreamSynchronize(s));
        if (herr) return fail(CURC_ERR_CUDA, "curc_pack_split_noalloc: bulk copy wait timed out");
        return CURC_OK;
    } catch (const std::exception& e) {
        return fail(CURC_ERR_CUDA, e.what());
    }
}
