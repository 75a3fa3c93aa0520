// Stable compaction in one launch, with the item count read on the device.
//
// Tiles of CP_TILE items are taken in order from an atomic counter; each
// tile ranks its kept items with warp ballots, publishes its count, and
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
template <class Keep, class Move>
__global__ void __launch_bounds__(CP_THREADS) compact_kernel(const uint32_t* __restrict__ n_dev,
                                                             uint32_t* __restrict__ n_out, Keep keep, Move move,
                                                             unsigned long long* tiles, uint32_t* counter,
                                                             uint32_t base, uint32_t epoch, uint32_t* err) {
    __shared__ uint32_t s_tile, s_excl, s_warp[CP_THREADS / 32];
    const uint32_t n = *n_dev;
    if (threadIdx.x == 0) {
        s_tile = atomicAdd(counter, 1u) - base;
        if (blockIdx.x == 0 && uint64_t(n) > uint64_t(gridDim.x) * CP_TILE) atomicExch(err, 2u);
    }
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint64_t start = uint64_t(tile) * CP_TILE;
    if (start >= n && tile != 0) return;  // beyond the items; nobody looks back at it
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t rank[CP_ITEMS];
    uint32_t kept = 0;  // bit r: item r of this thread is kept
    uint32_t local = 0;
#pragma unroll
    for (int r = 0; r < CP_ITEMS; ++r) {
        const uint64_t i = start + uint64_t(r) * CP_THREADS + threadIdx.x;
        const bool k = i < n && keep(uint32_t(i));
        const uint32_t b = __ballot_sync(0xFFFFFFFFu, k);
        if (lane == 0) s_warp[warp] = __popc(b);
        __syncthreads();
        uint32_t before = 0, total = 0;
#pragma unroll
        for (int w = 0; w < CP_THREADS / 32; ++w) {
            const uint32_t c = s_warp[w];
            before += w < int(warp) ? c : 0;
            total += c;
        }
        rank[r] = local + before + __popc(b & ((1u << lane) - 1u));
        kept |= uint32_t(k) << r;
        local += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        uint32_t excl = 0;
        if (tile == 0) {
            atomicExch(&tiles[0], cp_pack(epoch, 2, local));
        } else {
            atomicExch(&tiles[tile], cp_pack(epoch, 1, local));
            uint32_t j = tile - 1;
            bool ok = true;
            while (true) {
                uint64_t v = 0;
                uint32_t spins = 0;
                for (;;) {
                    v = *reinterpret_cast<volatile unsigned long long*>(&tiles[j]);
                    if ((v >> 34) == (epoch & 0x3FFFFFFFu) && ((v >> 32) & 3u) != 0) break;
                    if (++spins >= CP_WAIT_LIMIT) break;
                    __nanosleep(64);
                }
                if (spins >= CP_WAIT_LIMIT) {
                    atomicExch(err, 1u);
                    ok = false;
                    break;
                }
                excl += uint32_t(v);
                if (((v >> 32) & 3u) == 2u || j == 0) break;
                --j;
            }
            // published even after a wait ran out, so that no later tile waits
            // in turn (the result is then void and *err tells the host)
            (void)ok;
            atomicExch(&tiles[tile], cp_pack(epoch, 2, excl + local));
        }
        s_excl = excl;
        if (start + CP_TILE >= n) *n_out = excl + local;
    }
    __syncthreads();
    const uint32_t excl = s_excl;
#pragma unroll
    for (int r = 0; r < CP_ITEMS; ++r)
        if ((kept >> r) & 1u) move(uint32_t(start + uint64_t(r) * CP_THREADS + threadIdx.x), excl + rank[r]);
}

// Owns the tile states of a sequence of compactions on one stream.
class Compactor {
public:
    Compactor(uint32_t max_items, Arena& a, cudaStream_t s) : s_(s) {
        max_tiles_ = uint32_t(div_up(uint64_t(max_items ? max_items : 1), uint64_t(CP_TILE)));
        tiles_ = a.alloc<unsigned long long>(max_tiles_);
        counter_ = a.alloc<uint32_t>(2);
        err_ = counter_ + 1;
        CURC_CHECK(cudaMemsetAsync(tiles_, 0, size_t(max_tiles_) * 8, s));
        CURC_CHECK(cudaMemsetAsync(counter_, 0, 8, s));
    }
    // Compacts the first *n_dev (<= max_items) items; *n_out = number kept.
    template <class Keep, class Move>
    void run(const uint32_t* n_dev, uint32_t n_max, uint32_t* n_out, Keep keep, Move move) {
        const uint32_t grid = uint32_t(div_up(uint64_t(n_max ? n_max : 1), uint64_t(CP_TILE)));
        if (grid > max_tiles_) throw std::runtime_error("Compactor: more items than it was sized for");
        ++epoch_;
        compact_kernel<Keep, Move><<<grid, CP_THREADS, 0, s_>>>(n_dev, n_out, keep, move, tiles_, counter_, base_,
                                                                  epoch_, err_);
        CURC_LAUNCH_CHECK();
        base_ += grid;
    }
    // Fails if any wait ran out (reads one value back).
    void check() {
        if (read_scalar(err_, s_)) throw std::runtime_error("Compactor: a tile wait ran out");
    }

private:
    cudaStream_t s_;
    uint32_t max_tiles_ = 0, base_ = 0, epoch_ = 0;
    unsigned long long* tiles_ = nullptr;
    uint32_t* counter_ = nullptr;
    uint32_t* err_ = nullptr;
};

}  // namespace curc
