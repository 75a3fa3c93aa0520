// Device-wide primitives: arena, scan, stable compaction, stable radix sort.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <stdexcept>
#include <string>

#include <mutex>

#include "primitives.cuh"

namespace curc {

namespace {
std::atomic<uint64_t> g_launches{0};
}
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void count_launches(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
uint64_t launches() { return g_launches.load(); }

// ---------------------------------------------------------------- arena

Arena::~Arena() {
    for (auto& c : chunks_) cudaFree(c.base);
}

void* Arena::alloc_bytes(size_t bytes) {
    bytes = (bytes + 255) & ~size_t(255);
    if (bytes == 0) bytes = 256;
    while (cur_ < chunks_.size()) {
        Chunk& c = chunks_[cur_];
        if (c.used + bytes <= c.size) {
            void* p = c.base + c.used;
            c.used += bytes;
            high_water_ = std::max(high_water_, in_use());
            return p;
        }
        // chunks after the current one are free: take the first that is
        // large enough, moved up to follow the current one
        size_t fit = cur_ + 1;
        while (fit < chunks_.size() && chunks_[fit].size < bytes) ++fit;
        if (fit < chunks_.size()) {
            std::rotate(chunks_.begin() + cur_ + 1, chunks_.begin() + fit, chunks_.begin() + fit + 1);
            ++cur_;
            chunks_[cur_].used = 0;
            continue;
        }
        break;
    }
    size_t sz = std::max(bytes, chunk_);
    char* p = nullptr;
    if (cudaMalloc(&p, sz) != cudaSuccess) {
        // out of memory: give back the free chunks (all too small) and retry
        cudaGetLastError();
        const size_t keep = chunks_.empty() ? 0 : cur_ + 1;
        for (size_t i = keep; i < chunks_.size(); ++i) CURC_CHECK(cudaFree(chunks_[i].base));
        chunks_.resize(keep);
        if (cudaMalloc(&p, sz) != cudaSuccess) {
            cudaGetLastError();
            size_t held = 0, fr = 0, tot = 0;
            for (const auto& c : chunks_) held += c.size;
            cudaMemGetInfo(&fr, &tot);
            const std::string msg = "arena: out of device memory for " + std::to_string(sz >> 20) +
                                    " MiB (the arena holds " + std::to_string(held >> 20) + " MiB in " +
                                    std::to_string(chunks_.size()) + " chunks; " + std::to_string(fr >> 20) +
                                    " MiB free on the device)";
            throw CudaError(cudaErrorMemoryAllocation, msg.c_str());
        }
    }
    // keep chunks ordered as used: insert after the current one
    Chunk c{p, sz, bytes};
    if (chunks_.empty()) {
        chunks_.push_back(c);
        cur_ = 0;
    } else {
        chunks_.insert(chunks_.begin() + cur_ + 1, c);
        ++cur_;
        for (size_t i = cur_ + 1; i < chunks_.size(); ++i) chunks_[i].used = 0;
    }
    high_water_ = std::max(high_water_, in_use());
    return p;
}

size_t Arena::in_use() const {
    size_t u = 0;
    for (size_t i = 0; i <= cur_ && i < chunks_.size(); ++i) u += chunks_[i].used;
    return u;
}

void Arena::reset() {
    // Several chunks (blocks of changing sizes grew the arena): give them
    // back and keep one chunk that holds the largest run seen, so later runs
    // allocate nothing and chunks do not pile up.  Nothing is in use here.
    if (chunks_.size() > 1) {
        const size_t mib = size_t(1) << 20;
        const size_t need = std::max(chunk_, (high_water_ + mib - 1) / mib * mib);
        for (auto& c : chunks_) CURC_CHECK(cudaFree(c.base));
        chunks_.clear();
        char* p = nullptr;
        if (cudaMalloc(&p, need) == cudaSuccess)
            chunks_.push_back(Chunk{p, need, 0});
        else
            cudaGetLastError();  // no room for one chunk: allocate on demand again
    }
    for (auto& c : chunks_) c.used = 0;
    cur_ = 0;
}

void Arena::trim() {
    for (auto& c : chunks_) CURC_CHECK(cudaFree(c.base));
    chunks_.clear();
    cur_ = 0;
    high_water_ = 0;
}

void Arena::release(const Mark& m) {
    if (chunks_.empty()) return;
    for (size_t i = m.chunk + 1; i < chunks_.size(); ++i) chunks_[i].used = 0;
    cur_ = m.chunk;
    if (cur_ < chunks_.size()) chunks_[cur_].used = m.used;
}

// ---------------------------------------------------------------- small reads

namespace {
constexpr size_t READ_SMALL_MAX = 4096;

__global__ void read_small_kernel(const uint8_t* __restrict__ src, size_t bytes, uint8_t* dst) {
    for (size_t i = threadIdx.x; i < bytes; i += blockDim.x) dst[i] = src[i];
}

// Mapped pinned buffer of this host thread (portable: valid on every device
// through unified addressing), allocated on first use and kept until exit.
uint8_t* thread_readback_buffer() {
    thread_local struct Buf {
        uint8_t* p = nullptr;
        ~Buf() {
            if (p) cudaFreeHost(p);
        }
    } b;
    if (!b.p)
        CURC_CHECK(cudaHostAlloc(reinterpret_cast<void**>(&b.p), READ_SMALL_MAX,
                                 cudaHostAllocMapped | cudaHostAllocPortable));
    return b.p;
}
}  // namespace

void read_small(void* host, const void* dev, size_t bytes, cudaStream_t s) {
    if (bytes == 0) return;
    if (bytes > READ_SMALL_MAX) throw std::runtime_error("read_small: more than 4 KiB");
    uint8_t* buf = thread_readback_buffer();
    read_small_kernel<<<1, 128, 0, s>>>(static_cast<const uint8_t*>(dev), bytes, buf);
    CURC_LAUNCH_CHECK();
    CURC_CHECK(cudaStreamSynchronize(s));
    std::memcpy(host, buf, bytes);
}

// ---------------------------------------------------------------- pinned arena

PinnedArena::~PinnedArena() {
    for (auto& c : chunks_) cudaFreeHost(c.base);
}

PinnedArena& PinnedArena::operator=(PinnedArena&& o) noexcept {
    if (this != &o) {
        for (auto& c : chunks_) cudaFreeHost(c.base);
        chunks_ = std::move(o.chunks_);
        cur_ = o.cur_;
        o.chunks_.clear();
        o.cur_ = 0;
    }
    return *this;
}

uint8_t* PinnedArena::alloc(size_t bytes) {
    bytes = (bytes + 63) & ~size_t(63);
    while (cur_ < chunks_.size()) {
        Chunk& c = chunks_[cur_];
        if (c.used + bytes <= c.size) {
            uint8_t* p = c.base + c.used;
            c.used += bytes;
            return p;
        }
        ++cur_;
    }
    Chunk c{nullptr, std::max(bytes, size_t(256) << 20), 0};
    CURC_CHECK(cudaHostAlloc(reinterpret_cast<void**>(&c.base), c.size, cudaHostAllocPortable));
    c.used = bytes;
    chunks_.push_back(c);
    cur_ = chunks_.size() - 1;
    return c.base;
}

void PinnedArena::reset() {
    for (auto& c : chunks_) c.used = 0;
    cur_ = 0;
}

// ---------------------------------------------------------------- stage timer

size_t StageTimer::begin_span(const std::string& name) {
    Span sp{name, nullptr, nullptr};
    CURC_CHECK(cudaEventCreate(&sp.a));
    CURC_CHECK(cudaEventCreate(&sp.b));
    CURC_CHECK(cudaEventRecord(sp.a, s));
    ev.push_back(sp);
    return ev.size() - 1;
}

void StageTimer::end_span(size_t i) { CURC_CHECK(cudaEventRecord(ev[i].b, s)); }

void StageTimer::collect(std::map<std::string, float>& out) {
    CURC_CHECK(cudaStreamSynchronize(s));
    for (auto& e : ev) {
        float ms = 0;
        CURC_CHECK(cudaEventElapsedTime(&ms, e.a, e.b));
        out[e.name] += ms;
        cudaEventDestroy(e.a);
        cudaEventDestroy(e.b);
    }
    ev.clear();
    open.clear();
}

StageTimer*& active_timer() {
    thread_local StageTimer* t = nullptr;
    return t;
}

// ---------------------------------------------------------------- scan

namespace {
constexpr int SCAN_THREADS = 256, SCAN_ITEMS = 8, SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

template <class T>
__device__ T block_exclusive_sum(T v, T* block_total) {
    __shared__ T warp_sums[SCAN_THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        T w = lane < SCAN_THREADS / 32 ? warp_sums[lane] : T(0);
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            T y = __shfl_up_sync(0xFFFFFFFFu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < SCAN_THREADS / 32) warp_sums[lane] = w;
    }
    __syncthreads();
    T warp_prefix = warp ? warp_sums[warp - 1] : T(0);
    *block_total = warp_sums[SCAN_THREADS / 32 - 1];
    __syncthreads();
    return warp_prefix + x - v;
}

template <class T>
__global__ void __launch_bounds__(SCAN_THREADS) scan_reduce_kernel(const T* __restrict__ in, size_t n,
                                                                   T* __restrict__ sums) {
    const size_t base = size_t(blockIdx.x) * SCAN_TILE;
    T s = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        size_t idx = base + size_t(i) * SCAN_THREADS + threadIdx.x;
        if (idx < n) s += in[idx];
    }
    T total;
    block_exclusive_sum(s, &total);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

template <class T>
__global__ void __launch_bounds__(SCAN_THREADS) scan_apply_kernel(const T* in, T* out, size_t n,
                                                                  const T* __restrict__ offsets, T* total) {
    __shared__ T sm[SCAN_TILE];
    const size_t base = size_t(blockIdx.x) * SCAN_TILE;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        size_t idx = base + size_t(i) * SCAN_THREADS + threadIdx.x;
        sm[i * SCAN_THREADS + threadIdx.x] = idx < n ? in[idx] : T(0);
    }
    __syncthreads();
    T local[SCAN_ITEMS];
    T tsum = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        local[i] = sm[threadIdx.x * SCAN_ITEMS + i];
        tsum += local[i];
    }
    T btotal;
    T run = block_exclusive_sum(tsum, &btotal);
    if (offsets) run += offsets[blockIdx.x];
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        T t = local[i];
        sm[threadIdx.x * SCAN_ITEMS + i] = run;
        run += t;
    }
    if (total && gridDim.x == 1 && threadIdx.x == 0) *total = btotal;
    __syncthreads();
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        size_t idx = base + size_t(i) * SCAN_THREADS + threadIdx.x;
        if (idx < n) out[idx] = sm[i * SCAN_THREADS + threadIdx.x];
    }
}
}  // namespace

template <class T>
void exclusive_scan(const T* in, T* out, size_t n, T* total, Arena& a, cudaStream_t s) {
    if (n == 0) {
        if (total) CURC_CHECK(cudaMemsetAsync(total, 0, sizeof(T), s));
        return;
    }
    const size_t tiles = div_up(n, SCAN_TILE);
    if (tiles == 1) {
        scan_apply_kernel<T><<<1, SCAN_THREADS, 0, s>>>(in, out, n, nullptr, total);
        CURC_LAUNCH_CHECK();
        return;
    }
    auto m = a.mark();
    T* sums = a.alloc<T>(tiles);
    scan_reduce_kernel<T><<<unsigned(tiles), SCAN_THREADS, 0, s>>>(in, n, sums);
    CURC_LAUNCH_CHECK();
    exclusive_scan<T>(sums, sums, tiles, total, a, s);
    scan_apply_kernel<T><<<unsigned(tiles), SCAN_THREADS, 0, s>>>(in, out, n, sums, nullptr);
    CURC_LAUNCH_CHECK();
    a.release(m);
}

template void exclusive_scan<uint32_t>(const uint32_t*, uint32_t*, size_t, uint32_t*, Arena&, cudaStream_t);
template void exclusive_scan<uint64_t>(const uint64_t*, uint64_t*, size_t, uint64_t*, Arena&, cudaStream_t);

// ---------------------------------------------------------------- compaction

namespace {
constexpr int SEL_THREADS = 256, SEL_ITEMS = 8, SEL_TILE = SEL_THREADS * SEL_ITEMS;

__global__ void __launch_bounds__(SEL_THREADS) count_flags_kernel(const uint8_t* __restrict__ flags, size_t n,
                                                                  uint32_t* __restrict__ counts) {
    const size_t base = size_t(blockIdx.x) * SEL_TILE;
    uint32_t c = 0;
#pragma unroll
    for (int i = 0; i < SEL_ITEMS; ++i) {
        size_t idx = base + size_t(i) * SEL_THREADS + threadIdx.x;
        if (idx < n) c += flags[idx] != 0;
    }
    uint32_t total;
    block_exclusive_sum<uint32_t>(c, &total);
    if (threadIdx.x == 0) counts[blockIdx.x] = total;
}

template <class T, bool kIndices>
__global__ void __launch_bounds__(SEL_THREADS) select_kernel(const T* __restrict__ in, const uint8_t* __restrict__ flags,
                                                             size_t n, const uint32_t* __restrict__ offsets,
                                                             T* __restrict__ out) {
    // blocked arrangement: thread t owns tile items [t*ITEMS, (t+1)*ITEMS)
    const size_t base = size_t(blockIdx.x) * SEL_TILE + size_t(threadIdx.x) * SEL_ITEMS;
    uint8_t f[SEL_ITEMS];
    uint32_t c = 0;
#pragma unroll
    for (int i = 0; i < SEL_ITEMS; ++i) {
        size_t idx = base + i;
        f[i] = idx < n ? flags[idx] != 0 : 0;
        c += f[i];
    }
    uint32_t total;
    uint32_t pos = block_exclusive_sum<uint32_t>(c, &total) + offsets[blockIdx.x];
#pragma unroll
    for (int i = 0; i < SEL_ITEMS; ++i) {
        if (f[i]) {
            if constexpr (kIndices) out[pos] = T(base + i);
            else out[pos] = in[base + i];
            ++pos;
        }
    }
}

template <class T, bool kIndices>
void select_impl(const T* in, const uint8_t* flags, T* out, size_t n, uint32_t* count, Arena& a, cudaStream_t s) {
    if (n == 0) {
        CURC_CHECK(cudaMemsetAsync(count, 0, sizeof(uint32_t), s));
        return;
    }
    auto m = a.mark();
    const size_t tiles = div_up(n, SEL_TILE);
    uint32_t* off = a.alloc<uint32_t>(tiles);
    count_flags_kernel<<<unsigned(tiles), SEL_THREADS, 0, s>>>(flags, n, off);
    CURC_LAUNCH_CHECK();
    exclusive_scan<uint32_t>(off, off, tiles, count, a, s);
    select_kernel<T, kIndices><<<unsigned(tiles), SEL_THREADS, 0, s>>>(in, flags, n, off, out);
    CURC_LAUNCH_CHECK();
    a.release(m);
}
}  // namespace

template <class T>
void select_flagged(const T* in, const uint8_t* flags, T* out, size_t n, uint32_t* count, Arena& a, cudaStream_t s) {
    select_impl<T, false>(in, flags, out, n, count, a, s);
}
template void select_flagged<uint32_t>(const uint32_t*, const uint8_t*, uint32_t*, size_t, uint32_t*, Arena&,
                                       cudaStream_t);
template void select_flagged<uint64_t>(const uint64_t*, const uint8_t*, uint64_t*, size_t, uint32_t*, Arena&,
                                       cudaStream_t);

void select_indices(const uint8_t* flags, uint32_t* out, size_t n, uint32_t* count, Arena& a, cudaStream_t s) {
    select_impl<uint32_t, true>(nullptr, flags, out, n, count, a, s);
}

// ---------------------------------------------------------------- radix sort

namespace {
constexpr int RS_THREADS = 256, RS_ROUNDS = 16, RS_TILE = RS_THREADS * RS_ROUNDS, RS_WARPS = RS_THREADS / 32;

template <class K>
__device__ __forceinline__ uint32_t digit_of(K k, int shift, uint32_t mask) {
    return uint32_t(k >> shift) & mask;
}

template <class K>
__global__ void __launch_bounds__(RS_THREADS) rs_hist_kernel(const K* __restrict__ keys, size_t n, int shift,
                                                             uint32_t mask, uint32_t* __restrict__ hist,
                                                             uint32_t tiles) {
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const size_t base = size_t(blockIdx.x) * RS_TILE;
#pragma unroll 4
    for (int r = 0; r < RS_ROUNDS; ++r) {
        size_t idx = base + size_t(r) * RS_THREADS + threadIdx.x;
        if (idx < n) atomicAdd(&h[digit_of(keys[idx], shift, mask)], 1u);
    }
    __syncthreads();
    hist[size_t(threadIdx.x) * tiles + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter: items are ranked in index order.  Warp w takes the
// tile's items [512 w, 512 w + 512) in 16 rounds of 32 consecutive ones,
// keeping them in registers, and ranks each among the warp's earlier items
// of its digit with match_any and warp-private digit counters (no block
// barrier inside); the warps' counts are then scanned per digit, and the
// tile is reordered by digit in shared memory (its digit counts come from
// the scanned histogram: the difference of consecutive offsets) and written
// out in that order, so that items of one digit leave as one contiguous run
// and the stores coalesce.
template <class K, class V>
__global__ void __launch_bounds__(RS_THREADS) rs_scatter_kernel(const K* __restrict__ kin, const V* __restrict__ vin,
                                                                K* __restrict__ kout, V* __restrict__ vout, size_t n,
                                                                int shift, uint32_t mask,
                                                                const uint32_t* __restrict__ offsets, uint32_t tiles) {
    extern __shared__ __align__(16) uint8_t rs_smem[];
    K* sk = reinterpret_cast<K*>(rs_smem);
    V* sv = reinterpret_cast<V*>(rs_smem + sizeof(K) * RS_TILE);
    __shared__ uint32_t gbase[256];
    __shared__ uint32_t tstart[256];
    __shared__ uint32_t wcnt[RS_WARPS][256];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    {
        // this tile's count of digit tid, from the exclusive scan over
        // (digit, tile): the next flattened entry minus this one
        const size_t fi = size_t(tid) * tiles + blockIdx.x;
        const uint32_t g = offsets[fi];
        const uint32_t nx = fi + 1 < size_t(256) * tiles ? offsets[fi + 1] : uint32_t(n);
        gbase[tid] = g;
        tstart[tid] = nx - g;
    }
#pragma unroll
    for (int w = 0; w < RS_WARPS; ++w) wcnt[w][tid] = 0;
    __syncthreads();
    // exclusive scan of the tile's digit counts (256 entries, one per thread)
    {
        __shared__ uint32_t wsum[RS_WARPS];
        const uint32_t v = tstart[tid];
        uint32_t x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wsum[warp] = x;
        __syncthreads();
        uint32_t wbase = 0;
        for (int w = 0; w < warp; ++w) wbase += wsum[w];
        tstart[tid] = wbase + x - v;
    }
    const uint32_t lt_mask = (1u << lane) - 1u;
    const size_t base = size_t(blockIdx.x) * RS_TILE;
    const uint32_t items = uint32_t(min(size_t(RS_TILE), n - base));
    // this warp's items, ranked within the warp
    const size_t wb = base + size_t(warp) * (RS_TILE / RS_WARPS);
    uint32_t* cnt = wcnt[warp];
    K k[RS_ROUNDS];
    V v[RS_ROUNDS];
    uint32_t rk[RS_ROUNDS];
#pragma unroll
    for (int r = 0; r < RS_ROUNDS; ++r) {
        const size_t idx = wb + size_t(r) * 32 + lane;
        const bool valid = idx < n;
        k[r] = valid ? kin[idx] : K{};
        v[r] = (valid && vin) ? vin[idx] : V{};
        const uint32_t d = valid ? digit_of(k[r], shift, mask) : 256u;
        const uint32_t peers = __match_any_sync(0xFFFFFFFFu, d);
        const uint32_t before = __popc(peers & lt_mask);
        uint32_t c0 = 0;
        if (valid) c0 = cnt[d];  // the warp's earlier items of digit d
        __syncwarp();
        if (valid && before == 0) cnt[d] = c0 + __popc(peers);
        __syncwarp();
        rk[r] = c0 + before;
    }
    __syncthreads();
    // per digit: the items of earlier warps come first
    {
        uint32_t acc = 0;
#pragma unroll
        for (int w = 0; w < RS_WARPS; ++w) {
            const uint32_t c = wcnt[w][tid];
            wcnt[w][tid] = acc;
            acc += c;
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < RS_ROUNDS; ++r) {
        const size_t idx = wb + size_t(r) * 32 + lane;
        if (idx < n) {
            const uint32_t d = digit_of(k[r], shift, mask);
            const uint32_t lp = tstart[d] + cnt[d] + rk[r];
            sk[lp] = k[r];
            if (vin) sv[lp] = v[r];
        }
    }
    __syncthreads();
    // the tile in digit order: runs of one digit go to consecutive places
    for (uint32_t p = tid; p < items; p += RS_THREADS) {
        const K kk = sk[p];
        const uint32_t d = digit_of(kk, shift, mask);
        const uint32_t gpos = gbase[d] + (p - tstart[d]);
        kout[gpos] = kk;
        if (vout) vout[gpos] = sv[p];
    }
}

template <class K, class V>
constexpr size_t rs_smem_bytes() {
    return (sizeof(K) + sizeof(V)) * size_t(RS_TILE);
}

// The scatter kernel's dynamic shared-memory limit, raised once per device.
template <class K, class V>
void rs_prepare() {
    static std::mutex mu;
    static bool done[64] = {};
    int dev = 0;
    CURC_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) throw std::runtime_error("device ordinal out of range");
    std::lock_guard<std::mutex> g(mu);
    if (!done[dev]) {
        CURC_CHECK(cudaFuncSetAttribute(rs_scatter_kernel<K, V>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        int(rs_smem_bytes<K, V>())));
        done[dev] = true;
    }
}
}  // namespace

template <class K, class V>
void radix_sort_pairs(K* keys, V* vals, size_t n, int begin_bit, int end_bit, Arena& a, cudaStream_t s) {
    if (n <= 1 || end_bit <= begin_bit) return;
    if (n > 0xFFFFFFFFull) throw std::runtime_error("radix_sort_pairs: more than 2^32 items");
    auto m = a.mark();
    K* kalt = a.alloc<K>(n);
    V* valt = vals ? a.alloc<V>(n) : nullptr;
    const uint32_t tiles = uint32_t(div_up(n, RS_TILE));
    uint32_t* hist = a.alloc<uint32_t>(size_t(256) * tiles);
    K* kc = keys;
    V* vc = vals;
    rs_prepare<K, V>();
    for (int shift = begin_bit; shift < end_bit; shift += 8) {
        const int bits = std::min(8, end_bit - shift);
        const uint32_t mask = (1u << bits) - 1u;
        rs_hist_kernel<K><<<tiles, RS_THREADS, 0, s>>>(kc, n, shift, mask, hist, tiles);
        CURC_LAUNCH_CHECK();
        exclusive_scan<uint32_t>(hist, hist, size_t(256) * tiles, nullptr, a, s);
        K* ko = (kc == keys) ? kalt : keys;
        V* vo = vals ? ((vc == vals) ? valt : vals) : nullptr;
        rs_scatter_kernel<K, V><<<tiles, RS_THREADS, rs_smem_bytes<K, V>(), s>>>(kc, vc, ko, vo, n, shift, mask,
                                                                                 hist, tiles);
        CURC_LAUNCH_CHECK();
        kc = ko;
        vc = vo;
    }
    if (kc != keys) {
        CURC_CHECK(cudaMemcpyAsync(keys, kc, n * sizeof(K), cudaMemcpyDeviceToDevice, s));
        if (vals) CURC_CHECK(cudaMemcpyAsync(vals, vc, n * sizeof(V), cudaMemcpyDeviceToDevice, s));
    }
    a.release(m);
}

template void radix_sort_pairs<uint64_t, uint32_t>(uint64_t*, uint32_t*, size_t, int, int, Arena&, cudaStream_t);
template void radix_sort_pairs<uint32_t, uint32_t>(uint32_t*, uint32_t*, size_t, int, int, Arena&, cudaStream_t);
template void radix_sort_pairs<uint64_t, uint64_t>(uint64_t*, uint64_t*, size_t, int, int, Arena&, cudaStream_t);

// ---------------------------------------------------------------- misc

namespace {
__global__ void gather_words_kernel(const uint64_t* __restrict__ src, const uint32_t* __restrict__ idx, size_t n,
                                    int stride, int word, uint64_t* __restrict__ out) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        out[i] = src[size_t(idx[i]) * stride + word];
}

template <class T>
__global__ void fill_kernel(T* p, T v, size_t n) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        p[i] = v;
}

__global__ void iota_kernel(uint32_t* p, size_t n) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        p[i] = uint32_t(i);
}

int persistent_grid(size_t n) {
    size_t g = div_up(n, 256);
    return int(std::max<size_t>(1, std::min<size_t>(g, size_t(SM_COUNT_B200) * 16)));
}
}  // namespace

void gather_words(const uint64_t* src, const uint32_t* idx, size_t n, int stride, int word, uint64_t* out,
                  cudaStream_t s) {
    if (!n) return;
    gather_words_kernel<<<persistent_grid(n), 256, 0, s>>>(src, idx, n, stride, word, out);
    CURC_LAUNCH_CHECK();
}

template <class T>
void fill(T* p, T v, size_t n, cudaStream_t s) {
    if (!n) return;
    fill_kernel<T><<<persistent_grid(n), 256, 0, s>>>(p, v, n);
    CURC_LAUNCH_CHECK();
}
template void fill<uint8_t>(uint8_t*, uint8_t, size_t, cudaStream_t);
template void fill<uint16_t>(uint16_t*, uint16_t, size_t, cudaStream_t);
template void fill<uint32_t>(uint32_t*, uint32_t, size_t, cudaStream_t);
template void fill<uint64_t>(uint64_t*, uint64_t, size_t, cudaStream_t);

void iota(uint32_t* p, size_t n, cudaStream_t s) {
    if (!n) return;
    iota_kernel<<<persistent_grid(n), 256, 0, s>>>(p, n);
    CURC_LAUNCH_CHECK();
}

namespace {
// Marks elements that share their first word with a neighbour (tie runs).
__global__ void tie_flags_kernel(const uint64_t* __restrict__ k0, size_t n, uint8_t* __restrict__ tie) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint64_t v = k0[i];
    tie[i] = (i > 0 && k0[i - 1] == v) || (i + 1 < n && k0[i + 1] == v);
}

// 1 where a tie element starts a new run (its predecessor in the tie list
// is not its neighbour or has another first word).
__global__ void run_starts_kernel(const uint32_t* __restrict__ pos, const uint64_t* __restrict__ k0, uint32_t m,
                                  uint32_t* __restrict__ start) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m) return;
    start[t] = t == 0 || pos[t - 1] + 1 != pos[t] || k0[pos[t - 1]] != k0[pos[t]];
}

// inclusive count of run starts: equal for all elements of one run
__global__ void run_number_kernel(const uint32_t* __restrict__ excl, const uint32_t* __restrict__ start, uint32_t m,
                                  uint64_t* __restrict__ out) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < m) out[t] = uint64_t(excl[t]) + start[t];
}

__global__ void run_starts8_kernel(const uint32_t* __restrict__ pos, const uint64_t* __restrict__ k0, uint32_t m,
                                   uint8_t* __restrict__ start) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m) return;
    start[t] = t == 0 || pos[t - 1] + 1 != pos[t] || k0[pos[t - 1]] != k0[pos[t]];
}

// One warp per run of reads sharing their first word: runs of up to 32
// reads are ordered in place by their remaining words, ties by position
// (stable), each lane ranking its read against the others' words by
// shuffles.  Longer runs are flagged for the radix path.
__global__ void small_runs_kernel(const uint64_t* __restrict__ db, int W, uint32_t* __restrict__ ids,
                                  const uint32_t* __restrict__ pos, const uint32_t* __restrict__ rb, uint32_t R,
                                  uint32_t m, uint8_t* __restrict__ large) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < R; r += warps) {
        const uint32_t b = rb[r], e = r + 1 < R ? rb[r + 1] : m, len = e - b;
        if (len > 32) {
            for (uint32_t k = lane; k < len; k += 32) large[b + k] = 1;
            continue;
        }
        const uint32_t p0 = pos[b];
        uint32_t id = 0;
        uint64_t w[15];
#pragma unroll
        for (int k = 0; k < 15; ++k) w[k] = 0;
        if (lane < len) {
            id = ids[p0 + lane];
#pragma unroll
            for (int k = 0; k < 15; ++k)
                if (k + 1 < W) w[k] = db[uint64_t(id) * W + k + 1];
        }
        uint32_t rank = 0;
        for (uint32_t j = 0; j < len; ++j) {
            int c = 0;  // lane j's read against mine
#pragma unroll
            for (int k = 0; k < 15; ++k) {
                if (k + 1 < W) {
                    const uint64_t o = __shfl_sync(0xFFFFFFFFu, w[k], int(j));
                    if (c == 0 && o != w[k]) c = o < w[k] ? -1 : 1;
                }
            }
            rank += (c < 0 || (c == 0 && j < lane)) ? 1u : 0u;
        }
        __syncwarp();
        if (lane < len) ids[p0 + rank] = id;
        __syncwarp();
    }
}

__global__ void gather_ids_kernel(const uint32_t* __restrict__ ids, const uint32_t* __restrict__ pos, uint32_t m,
                                  uint32_t* __restrict__ out) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < m) out[t] = ids[pos[t]];
}

__global__ void scatter_ids_kernel(const uint32_t* __restrict__ vals, const uint32_t* __restrict__ pos, uint32_t m,
                                   uint32_t* __restrict__ ids) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < m) ids[pos[t]] = vals[t];
}
}  // namespace

void sort_ids_by_reads(const uint64_t* db, int W, int L, uint32_t* ids, size_t n, Arena& a, cudaStream_t s) {
    // Stable lexicographic order of the reads (compress.cu:1400-1407 under a
    // stable comparison sort; ties keep input order).  First by the first
    // 32 bases; then only the runs of reads that share them are ordered by
    // the remaining words: runs of up to 32 reads by one warp each, longer
    // runs by radix passes over the remaining words, least significant first,
    // and finally by run so that every run returns to its place.
    if (n <= 1) return;
    auto mk = a.mark();
    uint64_t* k0 = a.alloc<uint64_t>(n);
    {
        // the first-word sort alone (the tie runs below read counts back to the host)
        SubStage sp("sort_dedupe.first_word");
        gather_words(db, ids, n, W, 0, k0, s);
        const int lo0 = W == 1 ? 64 - 2 * L : 0;
        radix_sort_pairs<uint64_t, uint32_t>(k0, ids, n, lo0, 64, a, s);
    }
    if (W > 1) {
        uint8_t* tie = a.alloc<uint8_t>(n);
        tie_flags_kernel<<<grid_for(n, 256), 256, 0, s>>>(k0, n, tie);
        CURC_LAUNCH_CHECK();
        uint32_t* pos = a.alloc<uint32_t>(n);
        uint32_t* cnt = a.alloc<uint32_t>(1);
        select_indices(tie, pos, n, cnt, a, s);
        const uint32_t m0 = read_scalar(cnt, s);
        uint32_t m = 0;
        if (m0) {
            // runs of up to 32 reads: one warp each; longer runs: radix below
            uint8_t* st8 = a.alloc<uint8_t>(m0);
            run_starts8_kernel<<<grid_for(m0, 256), 256, 0, s>>>(pos, k0, m0, st8);
            CURC_LAUNCH_CHECK();
            uint32_t* rb = a.alloc<uint32_t>(m0);
            uint32_t* rc = a.alloc<uint32_t>(2);
            select_indices(st8, rb, m0, rc, a, s);
            const uint32_t R = read_scalar(rc, s);
            uint8_t* large = a.alloc<uint8_t>(m0);
            CURC_CHECK(cudaMemsetAsync(large, 0, m0, s));
            small_runs_kernel<<<grid_for(uint64_t(R) * 32, 256), 256, 0, s>>>(db, W, ids, pos, rb, R, m0, large);
            CURC_LAUNCH_CHECK();
            uint32_t* li = a.alloc<uint32_t>(m0);
            select_indices(large, li, m0, rc + 1, a, s);
            m = read_scalar(rc + 1, s);
            if (m) {
                uint32_t* lp = a.alloc<uint32_t>(m);
                gather_ids_kernel<<<grid_for(m, 256), 256, 0, s>>>(pos, li, m, lp);
                CURC_LAUNCH_CHECK();
                pos = lp;
            }
        }
        if (m) {
            uint32_t* sub = a.alloc<uint32_t>(m);
            uint64_t* key = a.alloc<uint64_t>(m);
            uint64_t* run = a.alloc<uint64_t>(m);
            gather_ids_kernel<<<grid_for(m, 256), 256, 0, s>>>(ids, pos, m, sub);
            CURC_LAUNCH_CHECK();
            {
                // run number = number of run starts before the element
                uint32_t* st = a.alloc<uint32_t>(m);
                uint32_t* ex = a.alloc<uint32_t>(m);
                run_starts_kernel<<<grid_for(m, 256), 256, 0, s>>>(pos, k0, m, st);
                CURC_LAUNCH_CHECK();
                exclusive_scan<uint32_t>(st, ex, m, nullptr, a, s);
                run_number_kernel<<<grid_for(m, 256), 256, 0, s>>>(ex, st, m, run);
                CURC_LAUNCH_CHECK();
            }
            // the run numbers ride along as the sort moves the ids: sort pairs
            // of (key, index into sub) and permute both at the end
            uint32_t* perm = a.alloc<uint32_t>(m);
            iota(perm, m, s);
            uint32_t* tmp = a.alloc<uint32_t>(m);
            for (int w = W - 1; w >= 1; --w) {
                gather_ids_kernel<<<grid_for(m, 256), 256, 0, s>>>(sub, perm, m, tmp);  // current order's ids
                CURC_LAUNCH_CHECK();
                gather_words(db, tmp, m, W, w, key, s);
                const int lo = w == W - 1 ? 64 - 2 * (L - 32 * (W - 1)) : 0;
                radix_sort_pairs<uint64_t, uint32_t>(key, perm, m, lo, 64, a, s);
            }
            // stable by run number (ascending with position)
            uint64_t* rk = a.alloc<uint64_t>(m);
            gather_words(run, perm, m, 1, 0, rk, s);
            int bits = 1;
            while (bits < 64 && (1ull << bits) <= uint64_t(m) + 1) ++bits;
            radix_sort_pairs<uint64_t, uint32_t>(rk, perm, m, 0, bits, a, s);
            gather_ids_kernel<<<grid_for(m, 256), 256, 0, s>>>(sub, perm, m, tmp);
            CURC_LAUNCH_CHECK();
            scatter_ids_kernel<<<grid_for(m, 256), 256, 0, s>>>(tmp, pos, m, ids);
            CURC_LAUNCH_CHECK();
        }
    }
    a.release(mk);
}

}  // namespace curc
