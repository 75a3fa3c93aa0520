// Stable compaction in one launch, with the item count read on the device.
//
// Tiles of CP_TILE items are taken in order from an atomic counter; each
// tile ranks its kept items with one block scan, publishes its count, and
// finds its output offset by looking back over the tiles before it
// (decoupled look-back: a predecessor publishes its own count at once and
// its inclusive offset as soon as it knows it).  Because the count is read
// on the device, loops of data-dependent passes can be queued without a
// host round trip per pass.
//
// Waits on a predecessor are bounded; a wait that runs out sets *err (the
// caller checks it on the host and fails) instead of spinning forever.
// Tile states carry the launch's epoch, so the state array is never reset.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "common.cuh"
#include "primitives.cuh"

namespace curc {

constexpr int CP_THREADS = 512;
constexpr int CP_ITEMS = 8;
constexpr uint32_t CP_TILE = CP_THREADS * CP_ITEMS;
constexpr uint32_t CP_WAIT_LIMIT = 1u << 22;

__device__ __forceinline__ uint64_t cp_pack(uint32_t epoch, uint32_t flag, uint32_t v) {
    return uint64_t(epoch & 0x3FFFFFFFu) << 34 | uint64_t(flag) << 32 | v;
}

// keep(i) -> bool for item i < n; move(i, dst) places kept item i at dst.
// Each thread takes CP_ITEMS consecutive items; one block scan ranks them;
// warp 0 looks back over 32 predecessor tiles per step.
template <class Keep, class Move>
__global__ void __launch_bounds__(CP_THREADS) compact_kernel(const uint32_t* __restrict__ n_dev,
                                                             uint32_t* __restrict__ n_out, Keep keep, Move move,
                                                             unsigned long long* tiles, uint32_t* counter,
                                                             uint32_t base, uint32_t epoch_arg, uint32_t* err,
                                                             const uint32_t* __restrict__ epoch_dev) {
    __shared__ uint32_t s_tile, s_excl, s_warp[CP_THREADS / 32];
    const uint32_t n = *n_dev;
    const uint32_t epoch = epoch_dev ? *epoch_dev : epoch_arg;
    if (threadIdx.x == 0) {
        s_tile = atomicAdd(counter, 1u) - base;
        if (blockIdx.x == 0 && uint64_t(n) > uint64_t(gridDim.x) * CP_TILE) atomicExch(err, 2u);
    }
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint64_t start = uint64_t(tile) * CP_TILE;
    if (start >= n && tile != 0) return;  // beyond the items; nobody looks back at it
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint64_t first = start + uint64_t(threadIdx.x) * CP_ITEMS;
    uint32_t kept = 0;  // bit r: item first + r is kept
#pragma unroll
    for (int r = 0; r < CP_ITEMS; ++r) {
        const uint64_t i = first + r;
        if (i < n && keep(uint32_t(i))) kept |= 1u << r;
    }
    // block-wide exclusive scan of the per-thread counts
    const uint32_t mine = __popc(kept);
    uint32_t incl = mine;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, d);
        if (lane >= uint32_t(d)) incl += v;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    uint32_t before = 0, local = 0;
#pragma unroll
    for (int w = 0; w < CP_THREADS / 32; ++w) {
        const uint32_t c = s_warp[w];
        before += w < int(warp) ? c : 0;
        local += c;
    }
    const uint32_t rank = before + incl - mine;
    if (warp == 0) {
        uint32_t excl = 0;
        const uint32_t ep = epoch & 0x3FFFFFFFu;
        if (tile == 0) {
            if (lane == 0) atomicExch(&tiles[0], cp_pack(epoch, 2, local));
        } else {
            if (lane == 0) atomicExch(&tiles[tile], cp_pack(epoch, 1, local));
            // window of up to 32 predecessors: lane l reads tile (top - l)
            int64_t top = int64_t(tile) - 1;
            bool ok = true;
            while (true) {
                const int64_t j = top - int64_t(lane);
                uint64_t v = cp_pack(epoch, 2, 0);  // lanes past tile 0 add nothing
                uint32_t spins = 0;
                if (j >= 0) {
                    for (;;) {
                        v = *reinterpret_cast<volatile unsigned long long*>(&tiles[j]);
                        if ((v >> 34) == ep && ((v >> 32) & 3u) != 0) break;
                        if (++spins >= CP_WAIT_LIMIT) break;
                        __nanosleep(64);
                    }
                }
                if (__any_sync(0xFFFFFFFFu, spins >= CP_WAIT_LIMIT)) {
                    ok = false;
                    break;
                }
                // nearest lane holding an inclusive offset; sum the lanes
                // before it and itself
                const uint32_t inc = __ballot_sync(0xFFFFFFFFu, ((v >> 32) & 3u) == 2u);
                const int stop = inc ? __ffs(inc) - 1 : 32;
                uint32_t add = int(lane) <= stop ? uint32_t(v) : 0u;
#pragma unroll
                for (int d = 16; d > 0; d >>= 1) add += __shfl_xor_sync(0xFFFFFFFFu, add, d);
                excl += add;
                if (inc) break;
                top -= 32;
            }
            if (!ok && lane == 0) atomicExch(err, 1u);
            // published even after a wait ran out, so that no later tile waits
            // in turn (the result is then void and *err tells the host)
            if (lane == 0) atomicExch(&tiles[tile], cp_pack(epoch, 2, excl + local));
        }
        if (lane == 0) {
            s_excl = excl;
            if (start + CP_TILE >= n) *n_out = excl + local;
        }
    }
    __syncthreads();
    uint32_t d = s_excl + rank;
#pragma unroll
    for (int r = 0; r < CP_ITEMS; ++r)
        if ((kept >> r) & 1u) move(uint32_t(first + r), d++);
}

// Before a replayable compaction: a fresh epoch and tile counter.
static __global__ void cp_begin_kernel(uint32_t* counter, uint32_t* epoch) {
    *counter = 0;
    *epoch = *epoch + 1;
}

// Owns the tile states of a sequence of compactions on one stream.  A
// Compactor is used either through run() (epoch and tile base kept on the
// host, one launch per compaction) or through run_replayable() (kept on the
// device and advanced by a one-thread kernel, so the launches can be
// captured once and replayed from a graph), not both.
class Compactor {
public:
    Compactor(uint32_t max_items, Arena& a, cudaStream_t s) : s_(s) {
        max_tiles_ = uint32_t(div_up(uint64_t(max_items ? max_items : 1), uint64_t(CP_TILE)));
        tiles_ = a.alloc<unsigned long long>(max_tiles_);
        counter_ = a.alloc<uint32_t>(3);
        err_ = counter_ + 1;
        epoch_dev_ = counter_ + 2;
        CURC_CHECK(cudaMemsetAsync(tiles_, 0, size_t(max_tiles_) * 8, s));
        CURC_CHECK(cudaMemsetAsync(counter_, 0, 12, s));
    }
    // Compacts the first *n_dev (<= max_items) items; *n_out = number kept.
    template <class Keep, class Move>
    void run(const uint32_t* n_dev, uint32_t n_max, uint32_t* n_out, Keep keep, Move move) {
        const uint32_t grid = grid_for_items(n_max);
        ++epoch_;
        compact_kernel<Keep, Move><<<grid, CP_THREADS, 0, s_>>>(n_dev, n_out, keep, move, tiles_, counter_, base_,
                                                                  epoch_, err_, nullptr);
        CURC_LAUNCH_CHECK();
        base_ += grid;
    }
    // The same, replayable: two launches that refer to no host state.
    template <class Keep, class Move>
    void run_replayable(const uint32_t* n_dev, uint32_t n_max, uint32_t* n_out, Keep keep, Move move) {
        const uint32_t grid = grid_for_items(n_max);
        cp_begin_kernel<<<1, 1, 0, s_>>>(counter_, epoch_dev_);
        CURC_LAUNCH_CHECK();
        compact_kernel<Keep, Move><<<grid, CP_THREADS, 0, s_>>>(n_dev, n_out, keep, move, tiles_, counter_, 0, 0,
                                                                  err_, epoch_dev_);
        CURC_LAUNCH_CHECK();
    }
    // Fails if any wait ran out (reads one value back).
    void check() {
        if (read_scalar(err_, s_)) throw std::runtime_error("Compactor: a tile wait ran out");
    }

private:
    uint32_t grid_for_items(uint32_t n_max) const {
        const uint32_t grid = uint32_t(div_up(uint64_t(n_max ? n_max : 1), uint64_t(CP_TILE)));
        if (grid > max_tiles_) throw std::runtime_error("Compactor: more items than it was sized for");
        return grid;
    }
    cudaStream_t s_;
    uint32_t max_tiles_ = 0, base_ = 0, epoch_ = 0;
    unsigned long long* tiles_ = nullptr;
    uint32_t* counter_ = nullptr;
    uint32_t* err_ = nullptr;
    uint32_t* epoch_dev_ = nullptr;
};

}  // namespace curc
