// Shared device helpers for the CURC pseudogenome path on sm_100a.
//
// Packed reads: 2 bits per base, MSB-first inside little-endian u64 words,
// A=0 C=1 G=2 T=3 (any other symbol packs as A), W = ceil(L/32) words per
// read, read i at words [i*W, (i+1)*W).  This is the reference's layout
// (compress.cu:2159-2174) so that every comparison of packed words orders
// reads exactly as the reference's comparators do.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>

namespace curc {

constexpr uint32_t INVALID = 0xFFFFFFFFu;   // constant.hpp:48
constexpr uint16_t INVALOFF = 0xFFFFu;      // constant.hpp:49
constexpr int SM_COUNT_B200 = 148;

struct CudaError : std::runtime_error {
    cudaError_t code;
    CudaError(cudaError_t c, const char* what) : std::runtime_error(what), code(c) {}
};

#define CURC_CHECK(expr)                                                                      \
    do {                                                                                      \
        cudaError_t e__ = (expr);                                                             \
        if (e__ != cudaSuccess) {                                                             \
            char b__[512];                                                                    \
            std::snprintf(b__, sizeof(b__), "%s failed: %s (%s:%d)", #expr, cudaGetErrorString(e__), \
                          __FILE__, __LINE__);                                                \
            throw ::curc::CudaError(e__, b__);                                                \
        }                                                                                     \
    } while (0)

// Every kernel launch of the library goes through this check, which also
// counts it (curc_kernel_launches).
void count_launch();
// Adds the launches a graph made on the device (its kernels times its replays).
void count_launches(uint64_t n);
#define CURC_LAUNCH_CHECK()             \
    do {                                \
        ::curc::count_launch();         \
        CURC_CHECK(cudaGetLastError()); \
    } while (0)

__host__ __device__ inline uint64_t div_up(uint64_t a, uint64_t b) { return (a + b - 1) / b; }

// fmix64 finalizer of MurmurHash3 (util.cuh:82-89)
__host__ __device__ __forceinline__ uint64_t murmur64(uint64_t x) {
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdULL;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ULL;
    x ^= x >> 33;
    return x;
}

// Smallest power of two >= items within [2^24, 2^31] (util.cuh:72-80)
inline uint32_t hash_size_for(uint64_t items) {
    uint32_t hs;
    int order = 24;
    do {
        hs = 1u << order;
        ++order;
    } while (order <= 31 && hs < items);
    return hs;
}

// Bases [off, off+nb) of a packed read, first base most significant
// (util.cuh:180-188).  1 <= nb <= 32.
__device__ __forceinline__ uint64_t word_at(const uint64_t* __restrict__ r, uint32_t off, int nb) {
    const uint32_t w = off >> 5;
    const uint32_t s = (off & 31u) * 2u;
    uint64_t v = r[w] << s;
    if (64u - s < uint32_t(2 * nb)) v |= r[w + 1] >> (64u - s);
    return v >> (64 - 2 * nb);
}

// Same over a padded contiguous bit string (one zero word after the last
// base); util.cuh:189-195.
__device__ __forceinline__ uint64_t word_unaligned(const uint64_t* __restrict__ r, uint64_t off, int nb) {
    const uint64_t w = off >> 5;
    const uint32_t s = uint32_t(off & 31u) * 2u;
    uint64_t v = r[w] << s;
    if (s) v |= r[w + 1] >> (64u - s);
    return v >> (64 - 2 * nb);
}

__device__ __forceinline__ int code_at(const uint64_t* __restrict__ r, uint64_t off) {
    return int((r[off >> 5] >> (62 - 2 * (off & 31))) & 3u);
}

// Reverse complement of a k-mer held in the low 2k bits (util.cuh:220-226):
// complement, reverse the 2-bit groups of the whole word, keep the top k.
__device__ __forceinline__ uint64_t revcomp_kmer(uint64_t kmer, int k) {
    kmer = ~kmer;
    kmer = ((kmer & 0x3333333333333333ULL) << 2) | ((kmer & 0xCCCCCCCCCCCCCCCCULL) >> 2);
    kmer = ((kmer & 0x0F0F0F0F0F0F0F0FULL) << 4) | ((kmer & 0xF0F0F0F0F0F0F0F0ULL) >> 4);
    kmer = __byte_perm(uint32_t(kmer >> 32), 0, 0x0123) | (uint64_t(__byte_perm(uint32_t(kmer), 0, 0x0123)) << 32);
    return kmer >> (64 - 2 * k);
}

// Number of differing bases between two packed words (util.cuh:228-232).
__device__ __forceinline__ int base_mismatches(uint64_t a, uint64_t b) {
    uint64_t x = a ^ b;
    return __popcll(((x >> 1) | x) & 0x5555555555555555ULL);
}

__device__ __forceinline__ int ascii_code(uint8_t c) {
    // A/a 0, C/c 1, G/g 2, T/t 3, anything else 0 (base_encode_table & 3)
    switch (c) {
        case 'C': case 'c': return 1;
        case 'G': case 'g': return 2;
        case 'T': case 't': return 3;
        default: return 0;
    }
}

__device__ __forceinline__ char comp_char(char b) {  // util.cuh:152-164
    switch (b) {
        case 'a': return 't';
        case 'A': return 'T';
        case 'c': return 'g';
        case 'C': return 'G';
        case 'g': return 'c';
        case 'G': return 'C';
        case 't': return 'a';
        case 'T': return 'A';
        default: return 'N';
    }
}

// Three-way compare of read a[aoff, aoff+len) with read b[boff, boff+len),
// 32 bases at a time.
__device__ __forceinline__ int cmp_span(const uint64_t* a, uint32_t aoff, const uint64_t* b, uint32_t boff, int len) {
    for (int j = 0; j < len; j += 32) {
        const int nb = len - j < 32 ? len - j : 32;
        const uint64_t x = word_at(a, aoff + j, nb), y = word_at(b, boff + j, nb);
        if (x != y) return x < y ? -1 : 1;
    }
    return 0;
}

inline int grid_for(uint64_t n, int block, int per_thread = 1) {
    uint64_t g = div_up(n, uint64_t(block) * per_thread);
    if (g < 1) g = 1;
    if (g > 0x7FFFFFFFull) g = 0x7FFFFFFF;
    return int(g);
}

// Grid of a grid-stride kernel: as many blocks as stay resident on the
// device at once, no more than the n items need.
template <class K>
inline int resident_grid(K kernel, int block, uint64_t n) {
    int per_sm = 0;
    CURC_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, 0));
    const uint64_t cap = uint64_t(SM_COUNT_B200) * uint64_t(per_sm < 1 ? 1 : per_sm);
    const uint64_t need = div_up(n, uint64_t(block));
    return int(need < 1 ? 1 : (need < cap ? need : cap));
}

// Sum of a per-thread count over the block, added to *out with one atomic:
// a single global counter bumped by every warp serialises at the L2.  Every
// thread of the block calls it, after any divergent work.
template <class T>
__device__ __forceinline__ void block_tally(uint32_t v, T* out) {
    __shared__ uint32_t acc;
    if (threadIdx.x == 0) acc = 0;
    __syncthreads();
    v = __reduce_add_sync(0xFFFFFFFFu, v);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(&acc, v);
    __syncthreads();
    if (threadIdx.x == 0 && acc) atomicAdd(out, T(acc));
}

}  // namespace curc
