// a13: learned coder of the mismatch streams (no counterpart in the
// reference; the plain method is PPMd7 for bases and counts,
// compress.cu:1931-1933, and the CLR range coder for offsets,
// util.cuh:307-343).
//
// Per block the GPU lists the anchors of every record with mismatches (the
// start of the read and each mismatch) with their active input features and
// targets (gap to the next mismatch, read base at the mismatch).  Training
// is FP32 forward/backward/Adam with hand-written kernels (a tiled GEMM,
// bias/ReLU, softmax cross-entropy over the two output groups, column sums);
// the trained network is quantised to int8 weights, int32 accumulation and
// fixed-point requantisation (learned_model.hpp), and inference on the GPU
// runs the two dense layers on the tensor cores (tcgen05.mma kind::i8, s32
// accumulators in TMEM), which gives exactly the integers of the host
// reference, so the host decoder derives the same frequencies.
// The range-coded stream is split into chunks of records coded
// independently, so coding and the losslessness check run in parallel.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <random>

#include "../../include/curc_b200.h"
#include "block.cuh"
#include "host/host.hpp"
#include "learned_model.hpp"

namespace curc {
namespace learned {

// One anchor: active feature indices, targets, and the gap's valid maximum.
struct __align__(16) Anchor {
    uint8_t idx[20];
    uint8_t nidx;
    int8_t tbase;   // base outcome at this anchor's mismatch (-1: start anchor)
    int8_t tgap;    // gap bin to the next mismatch (-1: none)
    uint8_t strand; // the record's strand
    uint16_t gap;   // gap to the next mismatch
    uint16_t gmax;  // largest valid gap from this anchor
    uint32_t rec;   // record index
};
static_assert(sizeof(Anchor) == 32, "anchor layout");

constexpr int NPARAM = HID * IN + HID + HID * HID + HID + OUT * HID + OUT;

// Mismatch positions and bases of record r in pseudogenome order (as the
// emission kernel derives them).
__device__ int record_mismatches(const DevRecord& r, int m, int L, const uint64_t* db, int W, const uint8_t* nreads,
                                 const uint8_t* ref, const uint64_t* packed, uint16_t* pos, char* rbase) {
    int found = 0;
    if (!r.is_n) {
        const uint64_t* rd = db + uint64_t(r.read_id) * W;
        for (int p0 = 0; p0 < L; p0 += 32) {
            const int nb = L - p0 < 32 ? L - p0 : 32;
            const uint64_t gw = word_unaligned(packed, r.pos + p0, nb);
            const uint64_t rw = r.strand == 0 ? word_at(rd, p0, nb) : revcomp_kmer(word_at(rd, L - p0 - nb, nb), nb);
            uint64_t y = ((gw ^ rw) | ((gw ^ rw) >> 1)) & 0x5555555555555555ull;
            while (y) {
                const int bit = 63 - __clzll(y);
                y &= ~(1ull << bit);
                const int t = nb - 1 - bit / 2;
                if (found < m) {
                    pos[found] = uint16_t(p0 + t);
                    rbase[found] = "ACGT"[(rw >> (2 * (nb - 1 - t))) & 3u];
                }
                ++found;
            }
        }
    } else {
        const uint8_t* nd = nreads + uint64_t(r.read_id) * L;
        const uint8_t* g = ref + r.pos;
        for (int p = 0; p < L; ++p) {
            const int src = r.strand == 0 ? p : L - 1 - p;
            char rb = char(nd[src]);
            if (r.strand == 1) rb = comp_char(rb);
            if (char(g[p]) != rb) {
                if (found < m) {
                    pos[found] = uint16_t(p);
                    rbase[found] = rb;
                }
                ++found;
            }
        }
    }
    return found;
}

__global__ void anchor_count_kernel(const uint8_t* __restrict__ mis, uint32_t T, uint32_t* __restrict__ cnt) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < T) cnt[i] = mis[i] ? uint32_t(mis[i]) + 1u : 0u;
}

__global__ void anchors_kernel(const DevRecord* __restrict__ rec, const uint8_t* __restrict__ mis, uint32_t T,
                               const uint32_t* __restrict__ off, int L, const uint64_t* __restrict__ db, int W,
                               const uint8_t* __restrict__ nreads, const uint8_t* __restrict__ ref, uint64_t rl,
                               const uint64_t* __restrict__ packed, Anchor* __restrict__ out,
                               uint32_t* __restrict__ err) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= T || !mis[i]) return;
    const int m = mis[i];
    const DevRecord r = rec[i];
    uint16_t pos[104];
    char rb[104];
    if (m > 104 || record_mismatches(r, m, L, db, W, nreads, ref, packed, pos, rb) != m) {
        atomicExch(err, 1u);
        return;
    }
    Anchor* a = out + off[i];
    for (int j = 0; j <= m; ++j) {
        const int q = j == 0 ? -1 : pos[j - 1];
        const char pv = j >= 2 ? rb[j - 2] : 0;
        int idx[20];
        const int gmx = j < m ? L - 1 - q - (m - j) : 0;
        const int n = anchor_features(ref, rl, r.pos, q, L, r.strand, pv, m - j, gmx, idx);
        Anchor x;
        for (int t = 0; t < 20; ++t) x.idx[t] = t < n ? uint8_t(idx[t]) : 255;
        x.nidx = uint8_t(n);
        x.tbase = -1;
        if (j > 0) {
            const int o = base_outcome(char(ref[r.pos + q]), rb[j - 1]);
            if (o < 0) atomicExch(err, 2u);
            x.tbase = int8_t(o < 0 ? 0 : o);
        }
        if (j < m) {
            const int g = pos[j] - q - 1;
            x.gap = uint16_t(g);
            x.tgap = int8_t(gap_bin(g));
        } else {
            x.gap = 0;
            x.tgap = -1;
        }
        // the next mismatch leaves room for the m - j - 1 after it
        x.gmax = uint16_t(gmx);
        x.strand = r.strand;
        x.rec = i;
        a[j] = x;
    }
}

// ---------------------------------------------------------------- training

// C[m][n] = sum_k A(m,k) B(k,n) (+ C if acc); A(m,k) = A[m*sam + k*sak],
// B(k,n) = B[k*sbk + n*sbn].  32x32 tiles, one output per thread, k in
// order (deterministic).
__global__ void gemm_kernel(const float* __restrict__ A, const float* __restrict__ B, float* __restrict__ C, int M,
                            int N, int K, int sam, int sak, int sbk, int sbn, bool acc) {
    __shared__ float As[32][33], Bs[32][33];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8 threads, 4 rows each
    const int n = blockIdx.x * 32 + tx;
    float sum[4] = {0, 0, 0, 0};
    for (int k0 = 0; k0 < K; k0 += 32) {
        for (int r = ty; r < 32; r += 8) {
            const int mm = blockIdx.y * 32 + r, kk = k0 + tx;
            As[r][tx] = (mm < M && kk < K) ? A[size_t(mm) * sam + size_t(kk) * sak] : 0.f;
            const int kb = k0 + r;
            Bs[r][tx] = (kb < K && n < N) ? B[size_t(kb) * sbk + size_t(n) * sbn] : 0.f;
        }
        __syncthreads();
        for (int kk = 0; kk < 32; ++kk)
            for (int q = 0; q < 4; ++q) sum[q] += As[ty + 8 * q][kk] * Bs[kk][tx];
        __syncthreads();
    }
    for (int q = 0; q < 4; ++q) {
        const int mm = blockIdx.y * 32 + ty + 8 * q;
        if (mm < M && n < N) {
            float* c = C + size_t(mm) * N + n;
            *c = acc ? *c + sum[q] : sum[q];
        }
    }
}

void gemm(const float* A, const float* B, float* C, int M, int N, int K, int sam, int sak, int sbk, int sbn, bool acc,
          cudaStream_t s) {
    dim3 g((N + 31) / 32, (M + 31) / 32);
    gemm_kernel<<<g, 256, 0, s>>>(A, B, C, M, N, K, sam, sak, sbk, sbn, acc);
    CURC_LAUNCH_CHECK();
}

// dense one-hot inputs of a batch of anchors
__global__ void inputs_kernel(const Anchor* __restrict__ a, const uint32_t* __restrict__ sel, int B,
                              float* __restrict__ X) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    float* x = X + size_t(b) * IN;
    for (int i = 0; i < IN; ++i) x[i] = 0.f;
    const Anchor an = a[sel ? sel[b] : b];
    for (int t = 0; t < an.nidx; ++t) x[an.idx[t]] = 1.f;
}

__global__ void bias_act_kernel(float* __restrict__ H, const float* __restrict__ bias, int B, int N, bool relu) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= size_t(B) * N) return;
    float v = H[i] + bias[i % N];
    H[i] = relu ? fmaxf(v, 0.f) : v;
}

__global__ void relu_back_kernel(float* __restrict__ dH, const float* __restrict__ H, size_t n) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n && H[i] <= 0.f) dH[i] = 0.f;
}

// Cross-entropy of the base group (when the anchor has a base) and the gap
// group (when it has a next mismatch); dZ = (softmax - one-hot) / count.
__global__ void softmax_ce_kernel(const float* __restrict__ Z, const int8_t* __restrict__ tb,
                                  const int8_t* __restrict__ tg, int B, float inv_n, float* __restrict__ dZ,
                                  float* __restrict__ loss) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    const float* z = Z + size_t(b) * OUT;
    float* d = dZ + size_t(b) * OUT;
    float l = 0.f;
    for (int g = 0; g < 2; ++g) {
        const int o = g == 0 ? 0 : NB, k = g == 0 ? NB : NG;
        const int t = g == 0 ? tb[b] : tg[b];
        if (t < 0) {
            for (int j = 0; j < k; ++j) d[o + j] = 0.f;
            continue;
        }
        float mx = z[o];
        for (int j = 1; j < k; ++j) mx = fmaxf(mx, z[o + j]);
        float se = 0.f;
        for (int j = 0; j < k; ++j) se += expf(z[o + j] - mx);
        for (int j = 0; j < k; ++j) d[o + j] = (expf(z[o + j] - mx) / se - (j == t ? 1.f : 0.f)) * inv_n;
        l += (logf(se) + mx - z[o + t]) * inv_n;
    }
    loss[b] = l;
}

// out[n] = sum over rows of M (B x N), one thread per column, rows in order
__global__ void colsum_kernel(const float* __restrict__ M, int B, int N, float* __restrict__ out) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    float s = 0.f;
    for (int b = 0; b < B; ++b) s += M[size_t(b) * N + n];
    out[n] = s;
}

__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m1,
                            float* __restrict__ m2, int n, float lr, float b1, float b2, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    m1[i] = b1 * m1[i] + (1.f - b1) * gi;
    m2[i] = b2 * m2[i] + (1.f - b2) * gi * gi;
    p[i] -= lr * (m1[i] / c1) / (sqrtf(m2[i] / c2) + 1e-8f);
}

// ---------------------------------------------------------------- inference
//
// The int8 network on the 5th-generation tensor cores.  One CTA of 128
// threads takes 128 anchors at a time (one per thread and TMEM lane):
//   layer 1 (one-hot inputs): the sum of the anchor's weight columns, by the
//     thread itself, requantised to int8 and stored as the A operand;
//   layer 2: tcgen05.mma kind::i8, D[128 x 128] s32 in TMEM = A[128 x 128]
//     x W2^T, four K=32 steps issued by one thread; the thread of each
//     anchor reads its row back (tcgen05.ld), adds the bias, requantises and
//     stores it as the next A operand;
//   layer 3: the same with N = 32 (the OUT = 20 output rows of W3, zero
//     padded); each thread turns its logits into frequencies.
// Integer accumulation is exact in any order, so the frequencies equal the
// host model's (learned_model.hpp) bit for bit.  Operands live in shared
// memory in the no-swizzle K-major core-matrix layout: 8 rows x 16 bytes per
// 128-byte core matrix, the K chunks of a row group 128 bytes apart (leading
// byte offset) and row groups 1024 bytes apart (stride byte offset).  Waits
// on the MMA barrier are bounded: a wait that gives up sets the error word,
// and the CTA frees its TMEM and leaves.

constexpr int TC_ROWS = 128;                 // anchors per tile (MMA M)
constexpr int TC_N3 = 32;                    // padded output rows of layer 3
static_assert(OUT <= TC_N3, "layer 3 outputs exceed the padded MMA width");
constexpr int W1T_STRIDE = HID + 4;          // bytes per input row of W1^T (bank spread)
constexpr uint32_t TC_WAIT_LIMIT = 1u << 24;
constexpr uint32_t TC_TMEM_COLS = 128;

// Device copy of a model in the kernel's shared-memory layout.
struct TcModel {
    int8_t w1t[IN * W1T_STRIDE];             // W1 transposed: row = input feature
    int8_t w2[HID * HID];                    // B operand of layer 2, core-matrix layout
    int8_t w3[TC_N3 * HID];                  // B operand of layer 3, core-matrix layout
    int32_t b1[HID], b2[HID], b3[OUT];
    int32_t m1, sh1, m2, sh2, zmul, pad[3];
    uint32_t lut[LUTN];
};

// Byte offset of element (row r, k) of a K-major operand of 128 K bytes.
__host__ __device__ constexpr uint32_t core_off(int r, int k) {
    return uint32_t((r >> 3) * 1024 + (k >> 4) * 128 + (r & 7) * 16 + (k & 15));
}

TcModel tc_model(const Model& M) {
    TcModel t{};
    for (int i = 0; i < IN; ++i)
        for (int h = 0; h < HID; ++h) t.w1t[i * W1T_STRIDE + h] = M.w1[h][i];
    for (int h = 0; h < HID; ++h)
        for (int k = 0; k < HID; ++k) t.w2[core_off(h, k)] = M.w2[h][k];
    for (int o = 0; o < TC_N3; ++o)
        for (int k = 0; k < HID; ++k) t.w3[core_off(o, k)] = o < OUT ? M.w3[o][k] : int8_t(0);
    std::memcpy(t.b1, M.b1, sizeof(t.b1));
    std::memcpy(t.b2, M.b2, sizeof(t.b2));
    std::memcpy(t.b3, M.b3, sizeof(t.b3));
    t.m1 = M.m1;
    t.sh1 = M.sh1;
    t.m2 = M.m2;
    t.sh2 = M.sh2;
    t.zmul = M.zmul;
    std::memcpy(t.lut, M.lut, sizeof(t.lut));
    return t;
}

__device__ __forceinline__ uint32_t s_addr(const void* p) { return uint32_t(__cvta_generic_to_shared(p)); }

// Shared-memory matrix descriptor, no swizzle, K-major (version 1 for sm_100).
__device__ __forceinline__ uint64_t smem_desc(const void* base) {
    const uint64_t a = (s_addr(base) >> 4) & 0x3FFFu;
    const uint64_t lbo = 128u >> 4, sbo = 1024u >> 4;
    return a | (lbo << 16) | (sbo << 32) | (uint64_t(1) << 46);
}

// Instruction descriptor of kind::i8: s32 accumulator, signed A and B, both
// K-major, M = 128, N = n.
__host__ __device__ constexpr uint32_t idesc_i8(int n) {
    return (2u << 4) | (1u << 7) | (1u << 10) | (uint32_t(n >> 3) << 17) | (uint32_t(TC_ROWS >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        ::"r"(d), "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void tc_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(s_addr(bar))
                 : "memory");
}

__device__ __forceinline__ bool tc_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(s_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 32 consecutive 32-bit TMEM columns of this thread's lane.
__device__ __forceinline__ void tc_ld32(uint32_t taddr, int32_t* v) {
    uint32_t* r = reinterpret_cast<uint32_t*>(v);
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Bounded wait on the MMA barrier by every thread; false when it gave up.
__device__ __forceinline__ bool tc_wait_all(uint64_t* bar, uint32_t parity) {
    bool late = false;
    for (uint32_t w = 0; !tc_try_wait(bar, parity); ++w)
        if (w > TC_WAIT_LIMIT) {
            late = true;
            break;
        }
    return !__syncthreads_or(late);
}

constexpr size_t TC_SMEM = sizeof(TcModel) + TC_ROWS * HID + 1024;

__global__ void __launch_bounds__(TC_ROWS) infer_tc_kernel(const TcModel* __restrict__ gm,
                                                            const Anchor* __restrict__ a, uint32_t n,
                                                            uint16_t* __restrict__ freq, uint32_t* __restrict__ err) {
    extern __shared__ __align__(1024) uint8_t tc_smem[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_slot;
    // 1024-aligned operand tile, then the model
    uint8_t* base = tc_smem + ((1024u - (s_addr(tc_smem) & 1023u)) & 1023u);
    int8_t* A = reinterpret_cast<int8_t*>(base);
    TcModel& M = *reinterpret_cast<TcModel*>(base + TC_ROWS * HID);
    {
        const int words = sizeof(TcModel) / 16;
        const uint4* src = reinterpret_cast<const uint4*>(gm);
        uint4* dst = reinterpret_cast<uint4*>(&M);
        for (int i = threadIdx.x; i < words; i += blockDim.x) dst[i] = src[i];
    }
    const int tid = threadIdx.x, warp = tid >> 5;
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(s_addr(&bar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(s_addr(&tmem_slot)),
                     "r"(TC_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;
    const uint32_t lane_addr = tmem + (uint32_t(warp * 32) << 16);
    const uint32_t id2 = idesc_i8(HID), id3 = idesc_i8(TC_N3);
    uint32_t phase = 0;
    const uint32_t tiles = (n + TC_ROWS - 1) / TC_ROWS;
    for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x) {
        const uint32_t k = t * TC_ROWS + uint32_t(tid);
        const bool live = k < n;
        Anchor an{};
        if (live) an = a[k];
        // layer 1: sum of the active weight columns, 32 hidden units at a time
        for (int h0 = 0; h0 < HID; h0 += 32) {
            int32_t acc[32];
#pragma unroll
            for (int j = 0; j < 32; ++j) acc[j] = M.b1[h0 + j];
            for (int f = 0; f < (live ? int(an.nidx) : 0); ++f) {
                const int8_t* col = M.w1t + int(an.idx[f]) * W1T_STRIDE + h0;
#pragma unroll
                for (int j = 0; j < 32; j += 4) {
                    const char4 w = *reinterpret_cast<const char4*>(col + j);
                    acc[j] += w.x;
                    acc[j + 1] += w.y;
                    acc[j + 2] += w.z;
                    acc[j + 3] += w.w;
                }
            }
#pragma unroll
            for (int j = 0; j < 32; j += 16) {
                uint32_t v[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    uint32_t w = 0;
#pragma unroll
                    for (int b = 0; b < 4; ++b) w |= uint32_t(requant(acc[j + 4 * q + b], M.m1, M.sh1)) << (8 * b);
                    v[q] = w;
                }
                *reinterpret_cast<uint4*>(A + core_off(tid, h0 + j)) = make_uint4(v[0], v[1], v[2], v[3]);
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tc_fence_before();
        __syncthreads();
        // layer 2 on the tensor cores
        if (tid == 0) {
            tc_fence_after();
#pragma unroll
            for (int s = 0; s < HID / 32; ++s)
                tc_mma(tmem, smem_desc(A + s * 256), smem_desc(M.w2 + s * 256), id2, s > 0);
            tc_commit(&bar);
        }
        if (!tc_wait_all(&bar, phase)) {
            if (tid == 0) atomicExch(err, 1u);
            break;
        }
        phase ^= 1;
        tc_fence_after();
        // read back, bias, requantise: the A operand of layer 3
        for (int h0 = 0; h0 < HID; h0 += 32) {
            int32_t d[32];
            tc_ld32(lane_addr + uint32_t(h0), d);
#pragma unroll
            for (int j = 0; j < 32; j += 16) {
                uint32_t v[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    uint32_t w = 0;
#pragma unroll
                    for (int b = 0; b < 4; ++b) {
                        const int h = j + 4 * q + b;
                        w |= uint32_t(requant(d[h] + M.b2[h0 + h], M.m2, M.sh2)) << (8 * b);
                    }
                    v[q] = w;
                }
                *reinterpret_cast<uint4*>(A + core_off(tid, h0 + j)) = make_uint4(v[0], v[1], v[2], v[3]);
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tc_fence_before();
        __syncthreads();
        // layer 3 on the tensor cores (columns 0..31 again: layer 2's values are read)
        if (tid == 0) {
            tc_fence_after();
#pragma unroll
            for (int s = 0; s < HID / 32; ++s)
                tc_mma(tmem, smem_desc(A + s * 256), smem_desc(M.w3 + s * 256), id3, s > 0);
            tc_commit(&bar);
        }
        if (!tc_wait_all(&bar, phase)) {
            if (tid == 0) atomicExch(err, 1u);
            break;
        }
        phase ^= 1;
        tc_fence_after();
        int32_t z[32];
        tc_ld32(lane_addr, z);
        if (live) {
            int32_t zz[OUT];
#pragma unroll
            for (int o = 0; o < OUT; ++o) zz[o] = z[o] + M.b3[o];
            uint32_t fb[NB], fg[NG];
            logits_to_freq_lut(M.lut, M.zmul, zz, NB, NB, fb);
            logits_to_freq_lut(M.lut, M.zmul, zz + NB, gap_bin(an.gmax) + 1, NG, fg);
            uint16_t* f = freq + size_t(k) * OUT;
            for (int j = 0; j < NB; ++j) f[j] = uint16_t(fb[j]);
            for (int j = 0; j < NG; ++j) f[NB + j] = uint16_t(fg[j]);
        }
        tc_fence_before();
        __syncthreads();  // every lane read before the next tile's MMA overwrites TMEM
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS));
}

// ---------------------------------------------------------------- host side

struct Trainer {
    int device = 0;
    cudaStream_t s = nullptr;
    // training set (device)
    Anchor* anc = nullptr;
    size_t n = 0, cap = 0;
    // float parameters and Adam state (device)
    float *p = nullptr, *g = nullptr, *m1 = nullptr, *m2 = nullptr;
    Model model{};
    bool quantised = false;
    std::vector<uint8_t> stream;  // last encoded stream
    std::string err;

    Trainer() {
        CURC_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        CURC_CHECK(cudaMalloc(&p, NPARAM * 4));
        CURC_CHECK(cudaMalloc(&g, NPARAM * 4));
        CURC_CHECK(cudaMalloc(&m1, NPARAM * 4));
        CURC_CHECK(cudaMalloc(&m2, NPARAM * 4));
        init_params(1);
    }
    ~Trainer() {
        cudaFree(anc);
        cudaFree(p);
        cudaFree(g);
        cudaFree(m1);
        cudaFree(m2);
        if (s) cudaStreamDestroy(s);
    }
    // parameter offsets
    static constexpr size_t oW1 = 0, ob1 = oW1 + HID * IN, oW2 = ob1 + HID, ob2 = oW2 + HID * HID,
                            oW3 = ob2 + HID, ob3 = oW3 + OUT * HID;

    void init_params(uint64_t seed) {
        std::vector<float> h(NPARAM, 0.f);
        std::mt19937_64 rng(seed);
        auto fill = [&](size_t o, int fan_out, int fan_in) {
            std::normal_distribution<float> nd(0.f, std::sqrt(2.f / fan_in));
            for (size_t i = 0; i < size_t(fan_out) * fan_in; ++i) h[o + i] = nd(rng);
        };
        fill(oW1, HID, IN);
        fill(oW2, HID, HID);
        fill(oW3, OUT, HID);
        CURC_CHECK(cudaMemcpy(p, h.data(), NPARAM * 4, cudaMemcpyHostToDevice));
        CURC_CHECK(cudaMemset(m1, 0, NPARAM * 4));
        CURC_CHECK(cudaMemset(m2, 0, NPARAM * 4));
    }

    // forward + backward on B anchors with dense inputs X; grads to g
    void step(const float* X, const int8_t* tb, const int8_t* tg, int B, float* H1, float* H2, float* Z, float* dZ,
              float* dH2, float* dH1, float* lossv) {
        // forward: H1 = relu(X W1^T + b1), H2 = relu(H1 W2^T + b2), Z = H2 W3^T + b3
        gemm(X, p + oW1, H1, B, HID, IN, IN, 1, 1, IN, false, s);
        bias_act_kernel<<<grid_for(size_t(B) * HID, 256), 256, 0, s>>>(H1, p + ob1, B, HID, true);
        gemm(H1, p + oW2, H2, B, HID, HID, HID, 1, 1, HID, false, s);
        bias_act_kernel<<<grid_for(size_t(B) * HID, 256), 256, 0, s>>>(H2, p + ob2, B, HID, true);
        gemm(H2, p + oW3, Z, B, OUT, HID, HID, 1, 1, HID, false, s);
        bias_act_kernel<<<grid_for(size_t(B) * OUT, 256), 256, 0, s>>>(Z, p + ob3, B, OUT, false);
        CURC_LAUNCH_CHECK();
        softmax_ce_kernel<<<grid_for(B, 256), 256, 0, s>>>(Z, tb, tg, B, 1.f / float(B), dZ, lossv);
        CURC_LAUNCH_CHECK();
        // backward
        gemm(dZ, H2, g + oW3, OUT, HID, B, 1, OUT, HID, 1, false, s);  // dW3 = dZ^T H2
        colsum_kernel<<<grid_for(OUT, 128), 128, 0, s>>>(dZ, B, OUT, g + ob3);
        gemm(dZ, p + oW3, dH2, B, HID, OUT, OUT, 1, HID, 1, false, s);  // dH2 = dZ W3
        relu_back_kernel<<<grid_for(size_t(B) * HID, 256), 256, 0, s>>>(dH2, H2, size_t(B) * HID);
        gemm(dH2, H1, g + oW2, HID, HID, B, 1, HID, HID, 1, false, s);  // dW2 = dH2^T H1
        colsum_kernel<<<grid_for(HID, 128), 128, 0, s>>>(dH2, B, HID, g + ob2);
        gemm(dH2, p + oW2, dH1, B, HID, HID, HID, 1, HID, 1, false, s);  // dH1 = dH2 W2
        relu_back_kernel<<<grid_for(size_t(B) * HID, 256), 256, 0, s>>>(dH1, H1, size_t(B) * HID);
        gemm(dH1, X, g + oW1, HID, IN, B, 1, HID, IN, 1, false, s);  // dW1 = dH1^T X
        colsum_kernel<<<grid_for(HID, 128), 128, 0, s>>>(dH1, B, HID, g + ob1);
        CURC_LAUNCH_CHECK();
    }
};

}  // namespace learned
}  // namespace curc

using namespace curc;
using namespace curc::learned;

struct curc_learn {
    Trainer t;
};

namespace curc {
namespace learned {

// Anchors of a context's last block (device memory of `a`).
Anchor* block_anchors(Block& b, Arena& a, uint32_t* count_out) {
    const uint32_t T = b.n_records;
    uint32_t* cnt = a.alloc<uint32_t>(size_t(T) + 1);
    uint32_t* off = a.alloc<uint32_t>(size_t(T) + 1);
    uint32_t* tot = a.alloc<uint32_t>(2);
    CURC_CHECK(cudaMemsetAsync(tot, 0, 8, b.stream));
    if (T) {
        anchor_count_kernel<<<grid_for(T, 256), 256, 0, b.stream>>>(b.smis, T, cnt);
        CURC_LAUNCH_CHECK();
    }
    exclusive_scan<uint32_t>(cnt, off, T, tot, a, b.stream);
    const uint32_t na = read_scalar(tot, b.stream);
    Anchor* out = a.alloc<Anchor>(na ? na : 1);
    if (T) {
        anchors_kernel<<<grid_for(T, 128), 128, 0, b.stream>>>(b.srec, b.smis, T, off, b.p.L, b.db, b.p.W, b.nreads,
                                                               b.hq.seq, b.hq.len, b.hq.packed, out, tot + 1);
        CURC_LAUNCH_CHECK();
    }
    if (read_scalar(tot + 1, b.stream)) throw std::runtime_error("learned: mismatch recount disagrees");
    *count_out = na;
    return out;
}

// Frequencies of n anchors (device) from a quantised model, on the tensor
// cores.
void infer(const Model& model, const Anchor* a, uint32_t n, uint16_t* fq, Arena& ar, cudaStream_t s) {
    if (!n) return;
    static std::mutex mu;
    static bool attr[64] = {};
    int dev = 0;
    CURC_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) throw std::runtime_error("device ordinal out of range");
    {
        std::lock_guard<std::mutex> g(mu);
        if (!attr[dev]) {
            CURC_CHECK(cudaFuncSetAttribute(infer_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            int(TC_SMEM)));
            attr[dev] = true;
        }
    }
    const TcModel hm = tc_model(model);
    TcModel* dm = ar.alloc<TcModel>(1);
    uint32_t* err = ar.alloc<uint32_t>(1);
    CURC_CHECK(cudaMemcpyAsync(dm, &hm, sizeof(TcModel), cudaMemcpyHostToDevice, s));
    CURC_CHECK(cudaMemsetAsync(err, 0, 4, s));
    const uint32_t tiles = (n + TC_ROWS - 1) / TC_ROWS;
    const int grid = int(std::min<uint32_t>(tiles, uint32_t(SM_COUNT_B200) * 3));
    infer_tc_kernel<<<grid, TC_ROWS, TC_SMEM, s>>>(dm, a, n, fq, err);
    CURC_LAUNCH_CHECK();
    if (read_scalar(err, s)) throw std::runtime_error("learned: tensor-core wait timed out");
}

// The learned stream of a block (its anchors listed and the network run on
// the GPU, the range coding on the host, chunks of records in parallel).
std::string encode_stream(const Model& model, Block& b) {
    const int L = b.p.L;
    auto mk = b.arena.mark();
    uint32_t na = 0;
    Anchor* a = block_anchors(b, b.arena, &na);
    uint16_t* fq = b.arena.alloc<uint16_t>(size_t(na ? na : 1) * OUT);
    infer(model, a, na, fq, b.arena, b.stream);
    std::vector<Anchor> ha(na);
    std::vector<uint16_t> hf(size_t(na) * OUT);
    if (na) {
        CURC_CHECK(cudaMemcpyAsync(ha.data(), a, size_t(na) * sizeof(Anchor), cudaMemcpyDeviceToHost, b.stream));
        CURC_CHECK(cudaMemcpyAsync(hf.data(), fq, hf.size() * 2, cudaMemcpyDeviceToHost, b.stream));
    }
    CURC_CHECK(cudaStreamSynchronize(b.stream));
    b.arena.release(mk);
    // chunk boundaries: anchors of CHUNK_RECORDS records with mismatches
    std::vector<size_t> cut{0};
    uint32_t recs = 0;
    for (size_t k = 0; k < na; ++k)
        if (ha[k].tbase < 0 && k > 0 && ++recs % CHUNK_RECORDS == 0) cut.push_back(k);
    cut.push_back(na);
    const int nc = int(cut.size()) - 1;
    std::vector<std::string> chunks(nc);
    double bits[3] = {0, 0, 0};  // bases, gap bins, offsets inside bins
#pragma omp parallel for schedule(dynamic)
    for (int c = 0; c < nc; ++c) {
        RangeEncoder enc;
        BinModels bins;
        double cb[3] = {0, 0, 0};
        int q = -1;  // the anchor's offset along the read, in pseudogenome order
        for (size_t k = cut[c]; k < cut[c + 1]; ++k) {
            const Anchor& x = ha[k];
            const uint16_t* f = &hf[k * OUT];
            if (x.tbase < 0) q = -1;  // a record's start anchor
            if (x.tbase >= 0) {
                uint32_t cum = 0;
                for (int j = 0; j < x.tbase; ++j) cum += f[j];
                enc.encode(cum, f[x.tbase], TOTAL);
                cb[0] -= std::log2(double(f[x.tbase]) / TOTAL);
            }
            if (x.tgap >= 0) {
                uint32_t cum = 0;
                for (int j = 0; j < x.tgap; ++j) cum += f[NB + j];
                enc.encode(cum, f[NB + x.tgap], TOTAL);
                cb[1] -= std::log2(double(f[NB + x.tgap]) / TOTAL);
                const int lo = gap_bin_lo(x.tgap);
                const int hi = std::min(gap_bin_lo(x.tgap + 1), int(x.gmax) + 1);
                const int bc = bin_context(q, L, x.strand);
                uint32_t oc, of, ot;
                bins.lookup(bc, x.tgap, x.gap - lo, hi - lo, oc, of, ot);
                enc.encode(oc, of, ot);
                cb[2] -= std::log2(double(of) / ot);
                bins.update(bc, x.tgap, x.gap - lo);
                q += 1 + x.gap;
            }
        }
        chunks[c] = enc.finish();
#pragma omp critical
        for (int q = 0; q < 3; ++q) bits[q] += cb[q];
    }
    if (std::getenv("CURC_VERBOSE"))
        std::fprintf(stderr, "curc: learned bytes: bases %.0f, gap bins %.0f, offsets in bins %.0f (%u anchors)\n",
                     bits[0] / 8, bits[1] / 8, bits[2] / 8, na);
    std::string s;
    const uint32_t ncu = uint32_t(nc);
    s.append(reinterpret_cast<const char*>(&ncu), 4);
    for (auto& c : chunks) {
        const uint32_t len = uint32_t(c.size());
        s.append(reinterpret_cast<const char*>(&len), 4);
    }
    for (auto& c : chunks) s += c;
    return s;
}

}  // namespace learned
}  // namespace curc

namespace {

template <class F>
int guarded_learn(curc_learn* L, F&& f) {
    try {
        CURC_CHECK(cudaSetDevice(L->t.device));
        f();
        return CURC_OK;
    } catch (const CudaError& e) {
        L->t.err = e.what();
        return CURC_ERR_CUDA;
    } catch (const std::invalid_argument& e) {
        L->t.err = e.what();
        return CURC_ERR_ARG;
    } catch (const std::exception& e) {
        L->t.err = e.what();
        return CURC_ERR_STATE;
    }
}

// Quantises the float parameters (host copy) into the integer model, with
// activation scales from the largest activations over `calib` anchors.
void quantise(Trainer& T, const std::vector<float>& P, const std::vector<Anchor>& calib) {
    auto W1 = [&](int h, int i) { return P[Trainer::oW1 + size_t(h) * IN + i]; };
    auto W2 = [&](int h, int i) { return P[Trainer::oW2 + size_t(h) * HID + i]; };
    auto W3 = [&](int o, int i) { return P[Trainer::oW3 + size_t(o) * HID + i]; };
    auto amax = [](const float* w, size_t n) {
        float m = 1e-12f;
        for (size_t i = 0; i < n; ++i) m = std::max(m, std::fabs(w[i]));
        return m;
    };
    const float sw1 = amax(&P[Trainer::oW1], size_t(HID) * IN) / 127.f;
    const float sw2 = amax(&P[Trainer::oW2], size_t(HID) * HID) / 127.f;
    const float sw3 = amax(&P[Trainer::oW3], size_t(OUT) * HID) / 127.f;
    // float activations on the calibration set for the activation scales
    float mx1 = 1e-6f, mx2 = 1e-6f;
    std::vector<float> h1(HID), h2(HID);
    for (const Anchor& an : calib) {
        for (int h = 0; h < HID; ++h) {
            float v = P[Trainer::ob1 + h];
            for (int t = 0; t < an.nidx; ++t) v += W1(h, an.idx[t]);
            h1[h] = std::max(v, 0.f);
            mx1 = std::max(mx1, h1[h]);
        }
        for (int h = 0; h < HID; ++h) {
            float v = P[Trainer::ob2 + h];
            for (int t = 0; t < HID; ++t) v += W2(h, t) * h1[t];
            h2[h] = std::max(v, 0.f);
            mx2 = std::max(mx2, h2[h]);
        }
    }
    const float sa1 = mx1 / 127.f, sa2 = mx2 / 127.f;
    Model& M = T.model;
    auto q8 = [](float v) { return int8_t(std::max(-127.f, std::min(127.f, std::nearbyint(v)))); };
    for (int h = 0; h < HID; ++h) {
        for (int i = 0; i < IN; ++i) M.w1[h][i] = q8(W1(h, i) / sw1);
        M.b1[h] = int32_t(std::nearbyint(P[Trainer::ob1 + h] / sw1));
        for (int i = 0; i < HID; ++i) M.w2[h][i] = q8(W2(h, i) / sw2);
        M.b2[h] = int32_t(std::nearbyint(P[Trainer::ob2 + h] / (sa1 * sw2)));
    }
    for (int o = 0; o < OUT; ++o) {
        for (int i = 0; i < HID; ++i) M.w3[o][i] = q8(W3(o, i) / sw3);
        M.b3[o] = int32_t(std::nearbyint(P[Trainer::ob3 + o] / (sa2 * sw3)));
    }
    M.sh1 = M.sh2 = 24;
    M.m1 = int32_t(std::nearbyint(double(sw1) / sa1 * double(1 << 24)));
    M.m2 = int32_t(std::nearbyint(double(sa1) * sw2 / sa2 * double(1 << 24)));
    M.zmul = int32_t(std::nearbyint(double(sa2) * sw3 * 16.0 * 65536.0));
    if (M.zmul < 1) M.zmul = 1;
    for (int i = 0; i < LUTN; ++i)
        M.lut[i] = std::max<uint32_t>(1u, uint32_t(std::nearbyint(65536.0 * std::exp(-double(i) / 16.0))));
    T.quantised = true;
}

}  // namespace

extern "C" {

int curc_learn_create(int device, curc_learn** out) {
    if (!out) return CURC_ERR_ARG;
    *out = nullptr;
    try {
        CURC_CHECK(cudaSetDevice(device));
        auto* L = new curc_learn;
        L->t.device = device;
        *out = L;
        return CURC_OK;
    } catch (const std::exception& e) {
        curc::ctxless_error() = e.what();
        return CURC_ERR_CUDA;
    }
}

void curc_learn_destroy(curc_learn* L) {
    if (!L) return;
    cudaSetDevice(L->t.device);
    delete L;
}

const char* curc_learn_error(const curc_learn* L) { return L ? L->t.err.c_str() : ""; }

int curc_learn_add_block(curc_learn* L, curc_ctx* ctx) {
    if (!L || !ctx) return CURC_ERR_ARG;
    if (ctx)
        if (const int rc = curc::ctx_wait(ctx)) return rc;
    return guarded_learn(L, [&] {
        Block& b = *ctx->block;
        auto mk = b.arena.mark();
        uint32_t na = 0;
        Anchor* a = block_anchors(b, b.arena, &na);
        Trainer& T = L->t;
        if (T.n + na > T.cap) {
            const size_t cap = std::max(T.n + na, T.cap * 2 + 1024);
            Anchor* nb = nullptr;
            CURC_CHECK(cudaMalloc(&nb, cap * sizeof(Anchor)));
            if (T.n) CURC_CHECK(cudaMemcpyAsync(nb, T.anc, T.n * sizeof(Anchor), cudaMemcpyDeviceToDevice, b.stream));
            CURC_CHECK(cudaStreamSynchronize(b.stream));
            cudaFree(T.anc);
            T.anc = nb;
            T.cap = cap;
        }
        if (na) CURC_CHECK(cudaMemcpyAsync(T.anc + T.n, a, size_t(na) * sizeof(Anchor), cudaMemcpyDeviceToDevice, b.stream));
        CURC_CHECK(cudaStreamSynchronize(b.stream));
        T.n += na;
        b.arena.release(mk);
    });
}

uint64_t curc_learn_anchors(const curc_learn* L) { return L ? L->t.n : 0; }

int curc_learn_train(curc_learn* L, int epochs, int batch, float lr, uint64_t seed, float* final_loss) {
    if (!L || epochs < 1 || batch < 1) return CURC_ERR_ARG;
    return guarded_learn(L, [&] {
        Trainer& T = L->t;
        if (T.n == 0) throw std::runtime_error("learned: no training anchors");
        T.init_params(seed);
        const int B = int(std::min<size_t>(size_t(batch), T.n));
        float *X, *H1, *H2, *Z, *dZ, *dH2, *dH1, *lossv;
        int8_t *tb, *tg;
        uint32_t* sel;
        CURC_CHECK(cudaMalloc(&X, size_t(B) * IN * 4));
        CURC_CHECK(cudaMalloc(&H1, size_t(B) * HID * 4));
        CURC_CHECK(cudaMalloc(&H2, size_t(B) * HID * 4));
        CURC_CHECK(cudaMalloc(&dH1, size_t(B) * HID * 4));
        CURC_CHECK(cudaMalloc(&dH2, size_t(B) * HID * 4));
        CURC_CHECK(cudaMalloc(&Z, size_t(B) * OUT * 4));
        CURC_CHECK(cudaMalloc(&dZ, size_t(B) * OUT * 4));
        CURC_CHECK(cudaMalloc(&lossv, size_t(B) * 4));
        CURC_CHECK(cudaMalloc(&tb, B));
        CURC_CHECK(cudaMalloc(&tg, B));
        CURC_CHECK(cudaMalloc(&sel, size_t(B) * 4));
        std::vector<Anchor> ha(T.n);
        CURC_CHECK(cudaMemcpy(ha.data(), T.anc, T.n * sizeof(Anchor), cudaMemcpyDeviceToHost));
        std::vector<uint32_t> order(T.n);
        for (size_t i = 0; i < T.n; ++i) order[i] = uint32_t(i);
        std::mt19937_64 rng(seed);
        std::vector<int8_t> htb(B), htg(B);
        float last = 0.f;
        int step = 0;
        const float b1 = 0.9f, b2 = 0.999f;
        for (int e = 0; e < epochs; ++e) {
            std::shuffle(order.begin(), order.end(), rng);
            for (size_t s0 = 0; s0 + size_t(B) <= T.n; s0 += size_t(B)) {
                for (int b = 0; b < B; ++b) {
                    htb[b] = ha[order[s0 + b]].tbase;
                    htg[b] = ha[order[s0 + b]].tgap;
                }
                CURC_CHECK(cudaMemcpyAsync(sel, order.data() + s0, size_t(B) * 4, cudaMemcpyHostToDevice, T.s));
                CURC_CHECK(cudaMemcpyAsync(tb, htb.data(), B, cudaMemcpyHostToDevice, T.s));
                CURC_CHECK(cudaMemcpyAsync(tg, htg.data(), B, cudaMemcpyHostToDevice, T.s));
                inputs_kernel<<<grid_for(B, 128), 128, 0, T.s>>>(T.anc, sel, B, X);
                CURC_LAUNCH_CHECK();
                T.step(X, tb, tg, B, H1, H2, Z, dZ, dH2, dH1, lossv);
                ++step;
                adam_kernel<<<grid_for(NPARAM, 256), 256, 0, T.s>>>(
                    T.p, T.g, T.m1, T.m2, NPARAM, lr, b1, b2, 1.f - std::pow(b1, float(step)),
                    1.f - std::pow(b2, float(step)));
                CURC_LAUNCH_CHECK();
                CURC_CHECK(cudaStreamSynchronize(T.s));
            }
        }
        {  // mean loss of the last batch
            std::vector<float> lv(B);
            CURC_CHECK(cudaMemcpy(lv.data(), lossv, size_t(B) * 4, cudaMemcpyDeviceToHost));
            for (float v : lv) last += v;
        }
        for (void* q : {(void*)X, (void*)H1, (void*)H2, (void*)dH1, (void*)dH2, (void*)Z, (void*)dZ, (void*)lossv,
                        (void*)tb, (void*)tg, (void*)sel})
            cudaFree(q);
        if (final_loss) *final_loss = last;
        // quantise with up to 4096 anchors for calibration
        std::vector<float> P(NPARAM);
        CURC_CHECK(cudaMemcpy(P.data(), T.p, NPARAM * 4, cudaMemcpyDeviceToHost));
        std::vector<Anchor> calib;
        for (size_t i = 0; i < ha.size() && calib.size() < 4096; i += std::max<size_t>(1, ha.size() / 4096))
            calib.push_back(ha[i]);
        quantise(T, P, calib);
    });
}

int curc_learn_grad(curc_learn* L, const float* params, const float* x, const int8_t* tb, const int8_t* tg,
                    uint32_t n, float* loss, float* grads) {
    if (!L || !params || !x || !tb || !tg || !n || !loss || !grads) return CURC_ERR_ARG;
    return guarded_learn(L, [&] {
        Trainer& T = L->t;
        const int B = int(n);
        float *X, *H1, *H2, *Z, *dZ, *dH2, *dH1, *lossv;
        int8_t *dtb, *dtg;
        CURC_CHECK(cudaMalloc(&X, size_t(B) * IN * 4));
        CURC_CHECK(cudaMalloc(&H1, size_t(B) * HID * 4));
        CURC_CHECK(cudaMalloc(&H2, size_t(B) * HID * 4));
        CURC_CHECK(cudaMalloc(&dH1, size_t(B) * HID * 4));
        CURC_CHECK(cudaMalloc(&dH2, size_t(B) * HID * 4));
        CURC_CHECK(cudaMalloc(&Z, size_t(B) * OUT * 4));
        CURC_CHECK(cudaMalloc(&dZ, size_t(B) * OUT * 4));
        CURC_CHECK(cudaMalloc(&lossv, size_t(B) * 4));
        CURC_CHECK(cudaMalloc(&dtb, B));
        CURC_CHECK(cudaMalloc(&dtg, B));
        CURC_CHECK(cudaMemcpy(T.p, params, NPARAM * 4, cudaMemcpyHostToDevice));
        CURC_CHECK(cudaMemcpy(X, x, size_t(B) * IN * 4, cudaMemcpyHostToDevice));
        CURC_CHECK(cudaMemcpy(dtb, tb, B, cudaMemcpyHostToDevice));
        CURC_CHECK(cudaMemcpy(dtg, tg, B, cudaMemcpyHostToDevice));
        T.step(X, dtb, dtg, B, H1, H2, Z, dZ, dH2, dH1, lossv);
        CURC_CHECK(cudaStreamSynchronize(T.s));
        std::vector<float> lv(B);
        CURC_CHECK(cudaMemcpy(lv.data(), lossv, size_t(B) * 4, cudaMemcpyDeviceToHost));
        float l = 0.f;
        for (float v : lv) l += v;
        *loss = l;
        CURC_CHECK(cudaMemcpy(grads, T.g, NPARAM * 4, cudaMemcpyDeviceToHost));
        for (void* q : {(void*)X, (void*)H1, (void*)H2, (void*)dH1, (void*)dH2, (void*)Z, (void*)dZ, (void*)lossv,
                        (void*)dtb, (void*)dtg})
            cudaFree(q);
    });
}

uint64_t curc_learn_param_count(void) { return NPARAM; }

int curc_learn_model(curc_learn* L, const void** ptr, uint64_t* bytes) {
    if (!L || !ptr || !bytes) return CURC_ERR_ARG;
    if (!L->t.quantised) {
        L->t.err = "learned: no quantised model";
        return CURC_ERR_STATE;
    }
    *ptr = &L->t.model;
    *bytes = sizeof(Model);
    return CURC_OK;
}

int curc_learn_set_model(curc_learn* L, const void* ptr, uint64_t bytes) {
    if (!L || !ptr || bytes != sizeof(Model)) return CURC_ERR_ARG;
    std::memcpy(&L->t.model, ptr, sizeof(Model));
    L->t.quantised = true;
    return CURC_OK;
}

// Learned stream of the context's last block: a u32 chunk count, per chunk
// a u32 byte length, then the chunks (each an independent range-coded run
// over CHUNK_RECORDS records with mismatches).
int curc_learn_encode(curc_learn* L, curc_ctx* ctx, const void** out, uint64_t* bytes) {
    if (!L || !ctx || !out || !bytes) return CURC_ERR_ARG;
    if (ctx)
        if (const int rc = curc::ctx_wait(ctx)) return rc;
    return guarded_learn(L, [&] {
        Trainer& T = L->t;
        if (!T.quantised) throw std::runtime_error("learned: no quantised model");
        const std::string s = encode_stream(T.model, *ctx->block);
        T.stream.assign(s.begin(), s.end());
        *out = T.stream.data();
        *bytes = T.stream.size();
    });
}

// Runs the tensor-core inference over the context's last block and
// recomputes every anchor's frequencies with the host model
// (learned_model.hpp, the decoder's integers): *anchors receives the
// number of anchors and *mismatched how many differ in any frequency.
int curc_learn_infer_check(curc_learn* L, curc_ctx* ctx, uint64_t* anchors, uint64_t* mismatched) {
    if (!L || !ctx || !anchors || !mismatched) return CURC_ERR_ARG;
    if (ctx)
        if (const int rc = curc::ctx_wait(ctx)) return rc;
    return guarded_learn(L, [&] {
        Trainer& T = L->t;
        if (!T.quantised) throw std::runtime_error("learned: no quantised model");
        Block& b = *ctx->block;
        auto mk = b.arena.mark();
        uint32_t na = 0;
        Anchor* a = block_anchors(b, b.arena, &na);
        uint16_t* fq = b.arena.alloc<uint16_t>(size_t(na ? na : 1) * OUT);
        infer(T.model, a, na, fq, b.arena, b.stream);
        std::vector<Anchor> ha(na);
        std::vector<uint16_t> hf(size_t(na) * OUT);
        if (na) {
            CURC_CHECK(cudaMemcpyAsync(ha.data(), a, size_t(na) * sizeof(Anchor), cudaMemcpyDeviceToHost, b.stream));
            CURC_CHECK(cudaMemcpyAsync(hf.data(), fq, hf.size() * 2, cudaMemcpyDeviceToHost, b.stream));
        }
        CURC_CHECK(cudaStreamSynchronize(b.stream));
        b.arena.release(mk);
        uint64_t bad = 0;
#pragma omp parallel for reduction(+ : bad)
        for (int64_t k = 0; k < int64_t(na); ++k) {
            int idx[24];
            for (int t = 0; t < ha[k].nidx; ++t) idx[t] = ha[k].idx[t];
            uint32_t fb[NB], fg[NG];
            model_freqs(T.model, idx, ha[k].nidx, ha[k].gmax, fb, fg);
            const uint16_t* f = &hf[size_t(k) * OUT];
            bool same = true;
            for (int j = 0; j < NB; ++j) same &= f[j] == fb[j];
            for (int j = 0; j < NG; ++j) same &= f[NB + j] == fg[j];
            bad += same ? 0 : 1;
        }
        *anchors = na;
        *mismatched = bad;
    });
}

// Decodes a learned stream on the host (the integer model, features from the
// decoded positions and bases) and compares every gap and base with the
// context's last block.  *ok = 1 when all match.
int curc_learn_decode_check(curc_learn* L, curc_ctx* ctx, const void* data, uint64_t bytes, int* ok) {
    if (!L || !ctx || !data || !ok) return CURC_ERR_ARG;
    if (ctx)
        if (const int rc = curc::ctx_wait(ctx)) return rc;
    return guarded_learn(L, [&] {
        Trainer& T = L->t;
        Block& b = *ctx->block;
        auto mk = b.arena.mark();
        uint32_t na = 0;
        Anchor* a = block_anchors(b, b.arena, &na);
        std::vector<Anchor> ha(na);
        if (na) CURC_CHECK(cudaMemcpy(ha.data(), a, size_t(na) * sizeof(Anchor), cudaMemcpyDeviceToHost));
        b.arena.release(mk);
        // records, their mismatch counts and the pseudogenome on the host
        const uint32_t Tn = b.n_records;
        std::vector<DevRecord> rec(Tn);
        std::vector<uint8_t> mis(Tn), ref(b.hq.len);
        if (Tn) {
            CURC_CHECK(cudaMemcpy(rec.data(), b.srec, size_t(Tn) * sizeof(DevRecord), cudaMemcpyDeviceToHost));
            CURC_CHECK(cudaMemcpy(mis.data(), b.smis, Tn, cudaMemcpyDeviceToHost));
        }
        if (b.hq.len) CURC_CHECK(cudaMemcpy(ref.data(), b.hq.seq, b.hq.len, cudaMemcpyDeviceToHost));
        const int Lr = b.p.L;
        std::vector<uint64_t> pos(Tn), first(Tn);
        std::vector<uint8_t> strand(Tn);
        uint64_t total = 0;
        for (uint32_t r = 0; r < Tn; ++r) {
            pos[r] = rec[r].pos;
            strand[r] = rec[r].strand;
            first[r] = total;
            total += mis[r];
        }
        // what the block holds: offsets and bases from its anchors
        std::vector<uint16_t> toff(total), off(total);
        std::vector<char> tbase(total), base(total);
        for (size_t k = 0; k < na; ++k) {
            if (ha[k].tbase >= 0) continue;  // a record's start anchor
            const uint32_t r = ha[k].rec;
            int q = -1;
            for (int j = 0; j < mis[r]; ++j) {
                q += 1 + ha[k + j].gap;
                toff[first[r] + j] = uint16_t(q);
                tbase[first[r] + j] = outcome_base(char(ref[pos[r] + uint64_t(q)]), ha[k + j + 1].tbase);
            }
        }
        // decoded by the host-compiled copy of the decoder (the one `curc -d` runs)
        const std::string why = host::learned_decode(&T.model, static_cast<const uint8_t*>(data), bytes,
                                                     ref.data(), ref.size(), Lr, Tn,
                                                     pos.data(), strand.data(), mis.data(), off.data(), base.data());
        *ok = why.empty() && off == toff && base == tbase ? 1 : 0;
    });
}

int curc_plain_mismatch_bytes(curc_ctx* ctx, uint64_t* out) {
    if (!ctx || !out) return CURC_ERR_ARG;
    if (ctx)
        if (const int rc = curc::ctx_wait(ctx)) return rc;
    try {
        const Block& b = *ctx->block;
        host::BlockView v;
        v.reads_count = b.n;
        v.read_len = b.p.L;
        v.preserve_order = b.p.preserve_order;
        v.paired_end = b.p.paired_end;
        for (const auto& kv : b.host) v.streams[kv.first] = host::Buf{kv.second.ptr, kv.second.size};
        host::plain_mismatch_bytes(v, out);
        return CURC_OK;
    } catch (const std::exception& e) {
        ctx->err = e.what();
        return CURC_ERR_STATE;
    }
}

int curc_mismatch_general_bytes(curc_ctx* ctx, const char* bsc_path, const char* tmpdir, uint64_t* out) {
    if (!ctx || !bsc_path || !tmpdir || !out) return CURC_ERR_ARG;
    if (ctx)
        if (const int rc = curc::ctx_wait(ctx)) return rc;
    try {
        const Block& b = *ctx->block;
        host::BlockView v;
        v.reads_count = b.n;
        v.read_len = b.p.L;
        for (const auto& kv : b.host) v.streams[kv.first] = host::Buf{kv.second.ptr, kv.second.size};
        host::CoderParams cp;
        cp.bsc_path = bsc_path;
        cp.tmpdir = tmpdir;
        host::general_mismatch_bytes(v, cp, out);
        return CURC_OK;
    } catch (const std::exception& e) {
        ctx->err = e.what();
        return CURC_ERR_STATE;
    }
}

}  // extern "C"
