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
// uses dp4a over the packed int8 rows, which gives exactly the integers of
// the host reference, so the host decoder derives the same frequencies.
// The range-coded stream is split into chunks of records coded
// independently, so coding and the losslessness check run in parallel.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
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
    uint8_t pad0;
    uint16_t gap;   // gap to the next mismatch
    uint16_t gmax;  // largest valid gap from this anchor
    uint32_t rec;   // record index
};
static_assert(sizeof(Anchor) == 32, "anchor layout");

constexpr int NPARAM = HID * IN + HID + HID * HID + HID + OUT * HID + OUT;
constexpr int CHUNK_RECORDS = 16384;

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
        x.pad0 = 0;
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

// int8 network per anchor, the integers of model_freqs: the sparse first
// layer as column sums, the dense layers as dp4a over packed int8 rows.
__global__ void __launch_bounds__(128) infer_kernel(const Model* __restrict__ gm, const Anchor* __restrict__ a,
                                                    uint32_t n, uint16_t* __restrict__ freq) {
    __shared__ Model M;
    {
        const int words = sizeof(Model) / 4;
        const uint32_t* src = reinterpret_cast<const uint32_t*>(gm);
        uint32_t* dst = reinterpret_cast<uint32_t*>(&M);
        for (int i = threadIdx.x; i < words; i += blockDim.x) dst[i] = src[i];
    }
    __syncthreads();
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const Anchor an = a[k];
    int32_t a1p[HID / 4];  // layer-1 activations packed 4 per word (0..127)
    for (int h4 = 0; h4 < HID / 4; ++h4) {
        uint32_t w = 0;
        for (int q = 0; q < 4; ++q) {
            const int h = 4 * h4 + q;
            int32_t acc = M.b1[h];
            for (int t = 0; t < an.nidx; ++t) acc += M.w1[h][an.idx[t]];
            w |= uint32_t(requant(acc, M.m1, M.sh1)) << (8 * q);
        }
        a1p[h4] = int32_t(w);
    }
    int32_t a2p[HID / 4];
    for (int h4 = 0; h4 < HID / 4; ++h4) {
        uint32_t w = 0;
        for (int q = 0; q < 4; ++q) {
            const int h = 4 * h4 + q;
            const int32_t* row = reinterpret_cast<const int32_t*>(M.w2[h]);
            int32_t acc = M.b2[h];
#pragma unroll 8
            for (int t = 0; t < HID / 4; ++t) acc = __dp4a(row[t], a1p[t], acc);
            w |= uint32_t(requant(acc, M.m2, M.sh2)) << (8 * q);
        }
        a2p[h4] = int32_t(w);
    }
    int32_t z[OUT];
    for (int o = 0; o < OUT; ++o) {
        const int32_t* row = reinterpret_cast<const int32_t*>(M.w3[o]);
        int32_t acc = M.b3[o];
#pragma unroll 8
        for (int t = 0; t < HID / 4; ++t) acc = __dp4a(row[t], a2p[t], acc);
        z[o] = acc;
    }
    uint32_t fb[NB], fg[NG];
    logits_to_freq(M, z, NB, NB, fb);
    logits_to_freq(M, z + NB, gap_bin(an.gmax) + 1, NG, fg);
    uint16_t* f = freq + size_t(k) * OUT;
    for (int j = 0; j < NB; ++j) f[j] = uint16_t(fb[j]);
    for (int j = 0; j < NG; ++j) f[NB + j] = uint16_t(fg[j]);
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
    return guarded_learn(L, [&] {
        Trainer& T = L->t;
        if (!T.quantised) throw std::runtime_error("learned: no quantised model");
        Block& b = *ctx->block;
        auto mk = b.arena.mark();
        uint32_t na = 0;
        Anchor* a = block_anchors(b, b.arena, &na);
        Model* dm = b.arena.alloc<Model>(1);
        CURC_CHECK(cudaMemcpyAsync(dm, &T.model, sizeof(Model), cudaMemcpyHostToDevice, b.stream));
        uint16_t* fq = b.arena.alloc<uint16_t>(size_t(na ? na : 1) * OUT);
        if (na) {
            infer_kernel<<<grid_for(na, 128), 128, 0, b.stream>>>(dm, a, na, fq);
            CURC_LAUNCH_CHECK();
        }
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
            for (size_t k = cut[c]; k < cut[c + 1]; ++k) {
                const Anchor& x = ha[k];
                const uint16_t* f = &hf[k * OUT];
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
                    uint32_t oc, of, ot;
                    bins.lookup(x.tgap, x.gap - lo, hi - lo, oc, of, ot);
                    enc.encode(oc, of, ot);
                    cb[2] -= std::log2(double(of) / ot);
                    bins.update(x.tgap, x.gap - lo);
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
        T.stream.assign(s.begin(), s.end());
        *out = T.stream.data();
        *bytes = T.stream.size();
    });
}

// Decodes a learned stream on the host (the integer model, features from the
// decoded positions and bases) and compares every gap and base with the
// context's last block.  *ok = 1 when all match.
int curc_learn_decode_check(curc_learn* L, curc_ctx* ctx, const void* data, uint64_t bytes, int* ok) {
    if (!L || !ctx || !data || !ok) return CURC_ERR_ARG;
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
        // records with mismatches, in order, and their first anchor index
        std::vector<uint32_t> rlist, first;
        for (size_t k = 0; k < na; ++k)
            if (ha[k].tbase < 0) {
                rlist.push_back(ha[k].rec);
                first.push_back(uint32_t(k));
            }
        const uint8_t* p = static_cast<const uint8_t*>(data);
        if (bytes < 4) throw std::runtime_error("learned: short stream");
        uint32_t nc;
        std::memcpy(&nc, p, 4);
        const uint32_t expect = uint32_t((rlist.size() + CHUNK_RECORDS - 1) / CHUNK_RECORDS);
        if (nc != expect && !(nc == 1 && rlist.empty())) throw std::runtime_error("learned: chunk count mismatch");
        std::vector<uint64_t> coff(nc + 1);
        coff[0] = 4 + 4ull * nc;
        for (uint32_t c = 0; c < nc; ++c) {
            uint32_t len;
            std::memcpy(&len, p + 4 + 4 * c, 4);
            coff[c + 1] = coff[c] + len;
        }
        if (coff[nc] != bytes) throw std::runtime_error("learned: stream length mismatch");
        int bad = 0;
#pragma omp parallel for schedule(dynamic) reduction(+ : bad)
        for (int c = 0; c < int(nc); ++c) {
            RangeDecoder dec(p + coff[c], size_t(coff[c + 1] - coff[c]));
            BinModels bins;
            const size_t r0 = size_t(c) * CHUNK_RECORDS, r1 = std::min(rlist.size(), r0 + CHUNK_RECORDS);
            for (size_t ri = r0; ri < r1; ++ri) {
                const DevRecord& r = rec[rlist[ri]];
                const int m = mis[rlist[ri]];
                int q = -1;
                char prev = 0;  // read base decoded at the previous anchor
                for (int j = 0; j <= m; ++j) {
                    int idx[20];
                    const int gmx = j < m ? Lr - 1 - q - (m - j) : 0;
                    const int n =
                        anchor_features(ref.data(), ref.size(), r.pos, q, Lr, r.strand, prev, m - j, gmx, idx);
                    uint32_t fb[NB], fg[NG];
                    model_freqs(T.model, idx, n, gmx, fb, fg);
                    const Anchor& truth = ha[first[ri] + j];
                    if (j > 0) {
                        const uint32_t v = dec.peek(TOTAL);
                        uint32_t cum = 0;
                        int o = 0;
                        while (cum + fb[o] <= v) cum += fb[o++];
                        dec.consume(cum, fb[o]);
                        if (o != truth.tbase) ++bad;
                        prev = outcome_base(char(ref[r.pos + q]), o);
                    }
                    if (j < m) {
                        uint32_t v = dec.peek(TOTAL), cum = 0;
                        int gb = 0;
                        while (cum + fg[gb] <= v) cum += fg[gb++];
                        dec.consume(cum, fg[gb]);
                        const int lo = gap_bin_lo(gb), hi = std::min(gap_bin_lo(gb + 1), gmx + 1);
                        const int w = std::max(1, hi - lo);
                        uint32_t oc, of;
                        const uint32_t ov = dec.peek(bins.total(gb, w));
                        const int o = bins.find(gb, w, ov, oc, of);
                        dec.consume(oc, of);
                        bins.update(gb, o);
                        const int g = lo + o;
                        if (g != truth.gap) ++bad;
                        q = q + 1 + g;
                    }
                }
            }
        }
        *ok = bad == 0 ? 1 : 0;
    });
}

int curc_plain_mismatch_bytes(curc_ctx* ctx, uint64_t* out) {
    if (!ctx || !out) return CURC_ERR_ARG;
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

}  // extern "C"
