// sched.cu -- kernels of the learned contention predictor: features, the
// device-side key frequency table, the MLP's forward and backward passes
// (tiled FP32-accumulating GEMMs over BF16 weights), Adam, abort labels and
// the stable low/high-risk partition. No counterpart in the reference: gCCTB
// schedules transactions in index order only (benchmark_cpu/ycsb.cu:262-285).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "sched.cuh"

namespace gcc {
namespace sched {

namespace {

// ---------------------------------------------------------------------------
// Features and the frequency table
// ---------------------------------------------------------------------------

// Half-warp per transaction: lane i holds request i; lane l then counts the
// requests that fall into sketch bins 4l .. 4l+3 and writes them as one u64.
__global__ void k_features(const gcc_ycsb_tx *__restrict__ txs, uint64_t first, uint64_t n,
                           const uint32_t *__restrict__ freq, uint16_t *__restrict__ out) {
    const uint64_t gt = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t t = gt >> 4;
    const unsigned l = threadIdx.x & 15u;
    const bool live = t < n;
    unsigned bin = 64u, wr = 0u, hot = 0u;
    if (live) {
        const gcc_ycsb_tx *T = txs + first + t;
        const uint32_t cnt = (uint32_t)T->request_cnt;
        if (l < cnt && l < (unsigned)kMaxOps) {
            const int2 rq = *(const int2 *)&T->requests[l];
            const uint32_t key = (uint32_t)rq.y;
            bin = sketch_bin(key);
            wr = rq.x > 0 ? 0u : 1u;
            hot = heat(__ldg(freq + freq_slot(key)));
        }
    }
    unsigned c0 = 0, c1 = 0, c2 = 0, c3 = 0;
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const unsigned b = __shfl_sync(0xFFFFFFFFu, bin, (int)((threadIdx.x & 16u) | (unsigned)i));
        c0 += b == 4u * l;
        c1 += b == 4u * l + 1u;
        c2 += b == 4u * l + 2u;
        c3 += b == 4u * l + 3u;
    }
    unsigned wsum = wr, hsum = hot;
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) {
        wsum += __shfl_xor_sync(0xFFFFFFFFu, wsum, o, 16);
        hsum += __shfl_xor_sync(0xFFFFFFFFu, hsum, o, 16);
    }
    if (!live) return;
    uint16_t *row = out + t * kFeatStride;
    const unsigned long long v = (unsigned long long)c0 | ((unsigned long long)c1 << 16) |
                                 ((unsigned long long)c2 << 32) | ((unsigned long long)c3 << 48);
    *(unsigned long long *)(row + 4 * l) = v;
    if (l == 0) {
        uint4 tail = make_uint4(wsum | (hsum << 16), 0u, 0u, 0u);
        *(uint4 *)(row + kSketch) = tail;
    }
}

// Variable-length transactions: the half-warp walks the requests in chunks
// of 16 (lane l holds request 16c + l of chunk c).
__global__ void k_features_var(const uint32_t *__restrict__ tx_off,
                               const gcc_ycsb_req *__restrict__ reqs, uint64_t first, uint64_t n,
                               const uint32_t *__restrict__ freq, uint16_t *__restrict__ out) {
    const uint64_t gt = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t t = gt >> 4;
    const unsigned l = threadIdx.x & 15u;
    const bool live = t < n;
    uint32_t beg = 0, cnt = 0;
    if (live) {
        beg = __ldg(tx_off + first + t);
        cnt = __ldg(tx_off + first + t + 1) - beg;
    }
    // chunks of the longest transaction of the warp's two half-warps
    const uint32_t chunks = __reduce_max_sync(0xFFFFFFFFu, (cnt + 15u) / 16u);
    unsigned c0 = 0, c1 = 0, c2 = 0, c3 = 0, wsum = 0, hsum = 0;
    for (uint32_t c = 0; c < chunks; ++c) {
        const uint32_t i = 16u * c + l;
        unsigned bin = 64u;
        if (live && i < cnt) {
            const int2 rq = *(const int2 *)(reqs + beg + i);
            const uint32_t key = (uint32_t)rq.y;
            bin = sketch_bin(key);
            wsum += rq.x > 0 ? 0u : 1u;
            hsum += heat(__ldg(freq + freq_slot(key)));
        }
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            const unsigned b = __shfl_sync(0xFFFFFFFFu, bin, (int)((threadIdx.x & 16u) | (unsigned)k));
            c0 += b == 4u * l;
            c1 += b == 4u * l + 1u;
            c2 += b == 4u * l + 2u;
            c3 += b == 4u * l + 3u;
        }
    }
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) {
        wsum += __shfl_xor_sync(0xFFFFFFFFu, wsum, o, 16);
        hsum += __shfl_xor_sync(0xFFFFFFFFu, hsum, o, 16);
    }
    if (!live) return;
    uint16_t *row = out + t * kFeatStride;
    const unsigned long long v = (unsigned long long)c0 | ((unsigned long long)c1 << 16) |
                                 ((unsigned long long)c2 << 32) | ((unsigned long long)c3 << 48);
    *(unsigned long long *)(row + 4 * l) = v;
    if (l == 0) *(uint4 *)(row + kSketch) = make_uint4(wsum | (hsum << 16), 0u, 0u, 0u);
}

__global__ void k_freq_add_var(const uint32_t *__restrict__ tx_off,
                               const gcc_ycsb_req *__restrict__ reqs, uint64_t first, uint64_t n,
                               uint32_t *freq) {
    const uint64_t t = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 4;
    const unsigned l = threadIdx.x & 15u;
    if (t >= n) return;
    const uint32_t beg = __ldg(tx_off + first + t), end = __ldg(tx_off + first + t + 1);
    for (uint32_t i = beg + l; i < end; i += 16u)
        atomicAdd(freq + freq_slot(reqs[i].key), 1u);
}

__global__ void k_freq_decay(uint32_t *freq) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < kFreqSize) freq[i] >>= 1;
}

__global__ void k_freq_add(const gcc_ycsb_tx *__restrict__ txs, uint64_t first, uint64_t n,
                           uint32_t *freq) {
    const uint64_t gt = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t t = gt >> 4;
    const unsigned l = threadIdx.x & 15u;
    if (t >= n) return;
    const gcc_ycsb_tx *T = txs + first + t;
    if (l >= (uint32_t)T->request_cnt) return;
    const int2 rq = *(const int2 *)&T->requests[l];
    atomicAdd(freq + freq_slot((uint32_t)rq.y), 1u);
}

// Lock plan of each transaction (KParams::plan): half-warp per transaction,
// lane l holds request l with c = its key's counter in the frequency table.
// Requests with c >= thr are planned, ordered by (c, key) ascending so the
// hottest key is locked last; every transaction of the batch compares two
// keys the same way (one table snapshot), so the plans agree on a global
// order of the keys they share. At most kPlanMax are planned (the hottest).
__global__ void k_lock_plan(const gcc_ycsb_tx *__restrict__ txs, uint64_t first, uint64_t n,
                            const uint32_t *__restrict__ freq, uint32_t thr,
                            unsigned long long *__restrict__ plan) {
    const uint64_t t = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 4;
    const unsigned l = threadIdx.x & 15u;
    const bool live = t < n;
    uint32_t c = 0u, key = 0u;
    bool hot = false;
    if (live) {
        const gcc_ycsb_tx *T = txs + first + t;
        const uint64_t cnt = T->request_cnt;
        if ((uint64_t)l < cnt) {
            key = (uint32_t)T->requests[l].key;
            c = __ldg(freq + freq_slot(key));
            hot = c >= thr;
        }
    }
    // rank among the hot requests of the transaction by (c, key)
    unsigned rank = 0u, nhot = 0u;
    const unsigned seg = threadIdx.x & 16u;
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        const uint32_t cj = __shfl_sync(0xFFFFFFFFu, c, (int)(seg | (unsigned)j));
        const uint32_t kj = __shfl_sync(0xFFFFFFFFu, key, (int)(seg | (unsigned)j));
        const bool hj = __shfl_sync(0xFFFFFFFFu, hot ? 1 : 0, (int)(seg | (unsigned)j)) != 0;
        nhot += hj ? 1u : 0u;
        rank += (hj && (cj < c || (cj == c && kj < key))) ? 1u : 0u;
    }
    const unsigned keep = nhot < (unsigned)kPlanMax ? nhot : (unsigned)kPlanMax;
    unsigned long long v = 0ull;
    if (hot && rank >= nhot - keep) {
        const unsigned j = rank - (nhot - keep);
        v = (1ull << l) | ((unsigned long long)l << (20 + 4 * j));
    }
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) v |= __shfl_xor_sync(0xFFFFFFFFu, v, o, 16);
    if (live && l == 0) plan[first + t] = v | ((unsigned long long)keep << 16);
}

// ---------------------------------------------------------------------------
// Tiled GEMM: C[m][n] (=, or += across K splits) sum_k A(m,k) B(k,n), with
// A(m,k) = A[m*sam + k*sak] and B(k,n) = B[k*sbk + n*sbn]; operands are
// converted to FP32 on the way into shared memory (u16 features are scaled
// by 1/16, BF16 widened), products accumulate in FP32. 64x64 tiles, K steps
// of 16, 256 threads with 4x4 outputs each. Optional epilogue: + bias[n]
// (BF16) then ReLU. With gridDim.z > 1 each z slice adds its K range into C
// atomically (C zeroed first, no epilogue).
// ---------------------------------------------------------------------------
template <class T> __device__ __forceinline__ float to_f(T v);
template <> __device__ __forceinline__ float to_f<float>(float v) { return v; }
template <> __device__ __forceinline__ float to_f<__nv_bfloat16>(__nv_bfloat16 v) {
    return __bfloat162float(v);
}
template <> __device__ __forceinline__ float to_f<uint16_t>(uint16_t v) {
    return (float)v * kFeatScale;
}

constexpr int kTM = 64, kTN = 64, kTK = 16;

template <class TA, class TB>
__global__ void __launch_bounds__(256) k_gemm(int M, int N, int K, int kchunk,
                                              const TA *__restrict__ A, long sam, long sak,
                                              const TB *__restrict__ B, long sbk, long sbn,
                                              float *__restrict__ C, int ldc,
                                              const __nv_bfloat16 *__restrict__ bias, int relu) {
    __shared__ __align__(16) float As[kTK][kTM + 4];
    __shared__ __align__(16) float Bs[kTK][kTN + 4];
    const int m0 = blockIdx.y * kTM, n0 = blockIdx.x * kTN;
    const int k_beg = blockIdx.z * kchunk;
    const int k_end = min(K, k_beg + kchunk);
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    float acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0.f;
    for (int k0 = k_beg; k0 < k_end; k0 += kTK) {
        // 64x16 of A and 16x64 of B: 1024 elements each, 4 per thread
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int e = threadIdx.x + r * 256;
            const int am = e / kTK, ak = e % kTK;
            const int gm = m0 + am, gk = k0 + ak;
            As[ak][am] = (gm < M && gk < k_end) ? to_f<TA>(A[(long)gm * sam + (long)gk * sak]) : 0.f;
            const int bk = e / kTN, bn = e % kTN;
            const int gk2 = k0 + bk, gn = n0 + bn;
            Bs[bk][bn] = (gn < N && gk2 < k_end) ? to_f<TB>(B[(long)gk2 * sbk + (long)gn * sbn]) : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < kTK; ++kk) {
            const float4 av = *(const float4 *)&As[kk][ty * 4];
            const float4 bv = *(const float4 *)&Bs[kk][tx * 4];
            const float a[4] = {av.x, av.y, av.z, av.w};
            const float b[4] = {bv.x, bv.y, bv.z, bv.w};
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int gm = m0 + ty * 4 + i;
        if (gm >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int gn = n0 + tx * 4 + j;
            if (gn >= N) continue;
            float v = acc[i][j];
            if (gridDim.z > 1) {
                atomicAdd(C + (long)gm * ldc + gn, v);
            } else {
                if (bias) v += __bfloat162float(bias[gn]);
                if (relu) v = fmaxf(v, 0.f);
                C[(long)gm * ldc + gn] = v;
            }
        }
    }
}

template <class TA, class TB>
cudaError_t gemm(cudaStream_t st, int M, int N, int K, const TA *A, long sam, long sak,
                 const TB *B, long sbk, long sbn, float *C, int ldc,
                 const __nv_bfloat16 *bias, bool relu, int splits) {
    if (splits < 1) splits = 1;
    int kchunk = (K + splits - 1) / splits;
    kchunk = (kchunk + kTK - 1) / kTK * kTK;
    splits = (K + kchunk - 1) / kchunk;
    if (splits > 1) {
        // split-K slices add atomically into zeroed output rows
        if (ldc != N) return cudaErrorInvalidValue;
        cudaError_t e = cudaMemsetAsync(C, 0, (size_t)M * N * sizeof(float), st);
        if (e != cudaSuccess) return e;
    }
    dim3 grid((N + kTN - 1) / kTN, (M + kTM - 1) / kTM, splits);
    k_gemm<TA, TB><<<grid, 256, 0, st>>>(M, N, K, kchunk, A, sam, sak, B, sbk, sbn, C, ldc,
                                          splits > 1 ? nullptr : bias, (splits == 1 && relu) ? 1 : 0);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Output head, loss and elementwise backward pieces
// ---------------------------------------------------------------------------

// Warp per row: z = h2 . w3 + b3, p = sigmoid(z). With labels: dz = (p - y)
// * scale and loss += softplus(z) - y z (the BCE of p, computed stably).
__global__ void k_head(const float *__restrict__ h2, const __nv_bfloat16 *__restrict__ w,
                       uint64_t n, float *__restrict__ p, const uint8_t *__restrict__ y,
                       float scale, float *__restrict__ dz, float *__restrict__ loss) {
    const uint64_t row = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned lane = threadIdx.x & 31u;
    if (row >= n) return;
    const float4 hv = *(const float4 *)(h2 + row * kHid + lane * 4);
    const __nv_bfloat16 *w3 = w + kOffW3 + lane * 4;
    float z = hv.x * __bfloat162float(w3[0]) + hv.y * __bfloat162float(w3[1]) +
              hv.z * __bfloat162float(w3[2]) + hv.w * __bfloat162float(w3[3]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) z += __shfl_xor_sync(0xFFFFFFFFu, z, o);
    z += __bfloat162float(w[kOffB3]);
    if (lane != 0) return;
    const float pr = 1.0f / (1.0f + expf(-z));
    if (p) p[row] = pr;
    if (y) {
        const float yy = y[row] ? 1.0f : 0.0f;
        dz[row] = (pr - yy) * scale;
        const float sp = fmaxf(z, 0.f) + log1pf(expf(-fabsf(z)));
        atomicAdd(loss, sp - yy * z);
    }
}

// dh2[r][j] = dz[r] w3[j] [h2[r][j] > 0]
__global__ void k_bwd_h2(const float *__restrict__ dz, const __nv_bfloat16 *__restrict__ w,
                         const float *__restrict__ h2, uint64_t n, float *__restrict__ dh2) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * kHid) return;
    const uint64_t r = i / kHid;
    const int j = (int)(i % kHid);
    dh2[i] = h2[i] > 0.f ? dz[r] * __bfloat162float(w[kOffW3 + j]) : 0.f;
}

__global__ void k_relu_mask(float *__restrict__ d, const float *__restrict__ h, uint64_t n) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && !(h[i] > 0.f)) d[i] = 0.f;
}

// out[j] = sum_r M[r * cols + j]: one block per column, fixed reduction order.
__global__ void k_colsum(const float *__restrict__ M, uint64_t rows, int cols, float *out) {
    __shared__ float red[256];
    const int j = blockIdx.x;
    float s = 0.f;
    for (uint64_t r = threadIdx.x; r < rows; r += blockDim.x) s += M[r * cols + j];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[j] = red[0];
}

__global__ void k_adam(float *__restrict__ master, __nv_bfloat16 *__restrict__ w,
                       const float *__restrict__ g, float *__restrict__ m, float *__restrict__ v,
                       int n, float lr, float bc1, float bc2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float x = master[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
    master[i] = x;
    w[i] = __float2bfloat16_rn(x);
}

__global__ void k_to_bf16(const float *__restrict__ a, __nv_bfloat16 *__restrict__ b, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = __float2bfloat16_rn(a[i]);
}

__global__ void k_labels(const unsigned *__restrict__ ab, uint64_t first, uint64_t n,
                         uint8_t *__restrict__ y) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = ab[first + i] > 0u ? 1 : 0;
}

// ---------------------------------------------------------------------------
// Stable partition by predicted risk
// ---------------------------------------------------------------------------
constexpr int kPartBlock = 1024;

// per block: low count, sum of p, sum of p over the high part
__global__ void k_part_count(const float *__restrict__ p, uint64_t n, float thr,
                             uint32_t *cnt, float *sums) {
    __shared__ float s_all[32], s_hi[32];
    __shared__ unsigned s_lo[32];
    const uint64_t i = (uint64_t)blockIdx.x * kPartBlock + threadIdx.x;
    const float v = i < n ? p[i] : 0.f;
    const bool hi = i < n && v > thr;
    const bool lo = i < n && !hi;
    float a = v, h = hi ? v : 0.f;
    unsigned c = __popc(__ballot_sync(0xFFFFFFFFu, lo));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xFFFFFFFFu, a, o);
        h += __shfl_xor_sync(0xFFFFFFFFu, h, o);
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) { s_all[w] = a; s_hi[w] = h; s_lo[w] = c; }
    __syncthreads();
    if (threadIdx.x == 0) {
        float ta = 0.f, th = 0.f;
        unsigned tc = 0;
        for (int k = 0; k < kPartBlock / 32; ++k) { ta += s_all[k]; th += s_hi[k]; tc += s_lo[k]; }
        cnt[blockIdx.x] = tc;
        sums[2 * blockIdx.x] = ta;
        sums[2 * blockIdx.x + 1] = th;
    }
}

// one block: exclusive scan of low counts (and of high counts), totals
__global__ void k_part_scan(uint32_t *cnt, const float *sums, uint32_t nb, uint64_t n,
                            uint32_t *counts, float *totals) {
    if (threadIdx.x != 0) return;
    uint32_t acc = 0;
    float ta = 0.f, th = 0.f;
    for (uint32_t b = 0; b < nb; ++b) {
        const uint32_t c = cnt[b];
        cnt[b] = acc;
        acc += c;
        ta += sums[2 * b];
        th += sums[2 * b + 1];
    }
    counts[0] = acc;
    totals[0] = ta;
    totals[1] = th;
    (void)n;
}

__global__ void k_part_scatter(const float *__restrict__ p, uint64_t first, uint64_t n, float thr,
                               const uint32_t *__restrict__ lo_off,
                               const uint32_t *__restrict__ counts, uint32_t *__restrict__ order) {
    __shared__ unsigned s_lo[32], s_hi[32];
    const uint64_t i = (uint64_t)blockIdx.x * kPartBlock + threadIdx.x;
    const bool live = i < n;
    const bool hi = live && p[i] > thr;
    const bool lo = live && !hi;
    const unsigned lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    const unsigned below = (1u << lane) - 1u;
    const unsigned blo = __ballot_sync(0xFFFFFFFFu, lo), bhi = __ballot_sync(0xFFFFFFFFu, hi);
    if (lane == 0) { s_lo[w] = __popc(blo); s_hi[w] = __popc(bhi); }
    __syncthreads();
    unsigned plo = 0, phi = 0;
    for (unsigned k = 0; k < w; ++k) { plo += s_lo[k]; phi += s_hi[k]; }
    if (!live) return;
    const uint64_t blk0 = (uint64_t)blockIdx.x * kPartBlock;
    const uint32_t lo_before = lo_off[blockIdx.x];
    const uint32_t hi_before = (uint32_t)(blk0 - lo_before);  // positions before the block that are high
    if (lo) {
        order[lo_before + plo + __popc(blo & below)] = (uint32_t)(first + i);
    } else {
        order[counts[0] + hi_before + phi + __popc(bhi & below)] = (uint32_t)(first + i);
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// Predictor
// ---------------------------------------------------------------------------
Predictor::~Predictor() {
    if (dev >= 0) cudaSetDevice(dev);
    void *bufs[] = {master, w, grad, adam_m, adam_v, h1, h2, dh1, dh2, p, dz, loss, labels, feat, freq};
    for (void *b : bufs)
        if (b) cudaFree(b);
}

static cudaError_t realloc_dev(void **ptr, size_t bytes) {
    if (*ptr) cudaFree(*ptr);
    *ptr = nullptr;
    return cudaMalloc(ptr, bytes ? bytes : 16);
}

cudaError_t Predictor::init(int device, cudaStream_t st, uint64_t rows, uint64_t seed) {
    dev = device;
    stream = st;
    cudaError_t e;
    if ((e = realloc_dev((void **)&master, kParams * 4))) return e;
    if ((e = realloc_dev((void **)&w, kParams * 2))) return e;
    if ((e = realloc_dev((void **)&grad, kParams * 4))) return e;
    if ((e = realloc_dev((void **)&adam_m, kParams * 4))) return e;
    if ((e = realloc_dev((void **)&adam_v, kParams * 4))) return e;
    if ((e = realloc_dev((void **)&loss, 16))) return e;
    if ((e = realloc_dev((void **)&freq, (size_t)kFreqSize * 4))) return e;
    if ((e = reserve(rows))) return e;
    // He-uniform initial weights from a counter-based hash of (seed, index);
    // biases start at zero
    std::vector<float> h(kParams, 0.f);
    auto uni = [&](uint64_t i) {
        return (float)((double)(hash3(seed, i, 0x4D4C50ull) >> 11) * (1.0 / 9007199254740992.0)) * 2.f - 1.f;
    };
    const float a1 = std::sqrt(6.f / kIn), a2 = std::sqrt(6.f / kHid), a3 = std::sqrt(3.f / kHid);
    for (int i = 0; i < kIn * kHid; ++i) h[kOffW1 + i] = a1 * uni(kOffW1 + i);
    for (int i = 0; i < kHid * kHid; ++i) h[kOffW2 + i] = a2 * uni(kOffW2 + i);
    for (int i = 0; i < kHid; ++i) h[kOffW3 + i] = a3 * uni(kOffW3 + i);
    if ((e = set_weights(h.data()))) return e;
    if ((e = clear_freq())) return e;
    return cudaStreamSynchronize(stream);
}

cudaError_t Predictor::reserve(uint64_t rows) {
    if (rows <= cap) return cudaSuccess;
    cudaError_t e;
    if ((e = realloc_dev((void **)&h1, rows * kHid * 4))) return e;
    if ((e = realloc_dev((void **)&h2, rows * kHid * 4))) return e;
    if ((e = realloc_dev((void **)&dh1, rows * kHid * 4))) return e;
    if ((e = realloc_dev((void **)&dh2, rows * kHid * 4))) return e;
    if ((e = realloc_dev((void **)&p, rows * 4))) return e;
    if ((e = realloc_dev((void **)&dz, rows * 4))) return e;
    if ((e = realloc_dev((void **)&labels, rows))) return e;
    if ((e = realloc_dev((void **)&feat, rows * kFeatStride * 2))) return e;
    cap = rows;
    return cudaSuccess;
}

cudaError_t Predictor::set_weights(const float *host) {
    cudaError_t e = cudaMemcpyAsync(master, host, kParams * 4, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(adam_m, 0, kParams * 4, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(adam_v, 0, kParams * 4, stream);
    if (e != cudaSuccess) return e;
    steps = 0;
    k_to_bf16<<<(kParams + 255) / 256, 256, 0, stream>>>(master, w, kParams);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    return e;
}

cudaError_t Predictor::get_weights(float *host) {
    cudaError_t e = cudaMemcpyAsync(host, master, kParams * 4, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    return e;
}

cudaError_t Predictor::features(const gcc_ycsb_tx *txs, uint64_t first, uint64_t n, uint16_t *out) {
    if (n == 0) return cudaSuccess;
    const uint64_t threads = n * 16;
    k_features<<<(unsigned)((threads + 255) / 256), 256, 0, stream>>>(txs, first, n, freq, out);
    return cudaGetLastError();
}

cudaError_t Predictor::features_var(const uint32_t *tx_off, const gcc_ycsb_req *reqs,
                                    uint64_t first, uint64_t n, uint16_t *out) {
    if (n == 0) return cudaSuccess;
    const uint64_t threads = n * 16;
    k_features_var<<<(unsigned)((threads + 255) / 256), 256, 0, stream>>>(tx_off, reqs, first, n,
                                                                          freq, out);
    return cudaGetLastError();
}

cudaError_t Predictor::observe_var(const uint32_t *tx_off, const gcc_ycsb_req *reqs,
                                   uint64_t first, uint64_t n) {
    k_freq_decay<<<kFreqSize / 256, 256, 0, stream>>>(freq);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || n == 0) return e;
    const uint64_t threads = n * 16;
    k_freq_add_var<<<(unsigned)((threads + 255) / 256), 256, 0, stream>>>(tx_off, reqs, first, n,
                                                                          freq);
    return cudaGetLastError();
}

cudaError_t Predictor::observe(const gcc_ycsb_tx *txs, uint64_t first, uint64_t n) {
    k_freq_decay<<<kFreqSize / 256, 256, 0, stream>>>(freq);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || n == 0) return e;
    const uint64_t threads = n * 16;
    k_freq_add<<<(unsigned)((threads + 255) / 256), 256, 0, stream>>>(txs, first, n, freq);
    return cudaGetLastError();
}

cudaError_t Predictor::lock_plan(const gcc_ycsb_tx *txs, uint64_t first, uint64_t n, uint32_t thr,
                                 unsigned long long *plan) {
    if (n == 0) return cudaSuccess;
    const uint64_t threads = n * 16;
    k_lock_plan<<<(unsigned)((threads + 255) / 256), 256, 0, stream>>>(txs, first, n, freq, thr, plan);
    return cudaGetLastError();
}

cudaError_t Predictor::clear_freq() {
    return cudaMemsetAsync(freq, 0, (size_t)kFreqSize * 4, stream);
}

cudaError_t Predictor::forward(const uint16_t *f, uint64_t n, float *p_out) {
    if (n == 0) return cudaSuccess;
    if (n > cap) return cudaErrorInvalidValue;
    const int M = (int)n;
    cudaError_t e = gemm<uint16_t, __nv_bfloat16>(stream, M, kHid, kIn, f, kFeatStride, 1,
                                                  w + kOffW1, kHid, 1, h1, kHid, w + kOffB1,
                                                  true, 1);
    if (e == cudaSuccess)
        e = gemm<float, __nv_bfloat16>(stream, M, kHid, kHid, h1, kHid, 1, w + kOffW2, kHid, 1, h2,
                                       kHid, w + kOffB2, true, 1);
    if (e != cudaSuccess) return e;
    k_head<<<(unsigned)((n * 32 + 255) / 256), 256, 0, stream>>>(h2, w, n, p_out, nullptr, 0.f,
                                                                 nullptr, nullptr);
    return cudaGetLastError();
}

cudaError_t Predictor::gradient(const uint16_t *f, const uint8_t *y, uint64_t n) {
    if (n == 0) return cudaErrorInvalidValue;
    if (n > cap) return cudaErrorInvalidValue;
    const int M = (int)n;
    cudaError_t e = cudaMemsetAsync(loss, 0, 4, stream);
    if (e == cudaSuccess)
        e = gemm<uint16_t, __nv_bfloat16>(stream, M, kHid, kIn, f, kFeatStride, 1, w + kOffW1,
                                          kHid, 1, h1, kHid, w + kOffB1, true, 1);
    if (e == cudaSuccess)
        e = gemm<float, __nv_bfloat16>(stream, M, kHid, kHid, h1, kHid, 1, w + kOffW2, kHid, 1, h2,
                                       kHid, w + kOffB2, true, 1);
    if (e != cudaSuccess) return e;
    k_head<<<(unsigned)((n * 32 + 255) / 256), 256, 0, stream>>>(h2, w, n, p, y, 1.0f / (float)n,
                                                                 dz, loss);
    if ((e = cudaGetLastError())) return e;
    const int splits = std::max(1, std::min(64, M / 256));
    // output layer: dw3 = h2^T dz, db3 = sum dz
    if ((e = gemm<float, float>(stream, kHid, 1, M, h2, 1, kHid, dz, 1, 0, grad + kOffW3, 1,
                                nullptr, false, splits)))
        return e;
    k_colsum<<<1, 256, 0, stream>>>(dz, n, 1, grad + kOffB3);
    k_bwd_h2<<<(unsigned)((n * kHid + 255) / 256), 256, 0, stream>>>(dz, w, h2, n, dh2);
    if ((e = cudaGetLastError())) return e;
    // layer 2: dW2 = h1^T dh2, db2 = colsum dh2, dh1 = dh2 W2^T masked by h1 > 0
    if ((e = gemm<float, float>(stream, kHid, kHid, M, h1, 1, kHid, dh2, kHid, 1, grad + kOffW2,
                                kHid, nullptr, false, splits)))
        return e;
    k_colsum<<<kHid, 256, 0, stream>>>(dh2, n, kHid, grad + kOffB2);
    if ((e = gemm<float, __nv_bfloat16>(stream, M, kHid, kHid, dh2, kHid, 1, w + kOffW2, 1, kHid,
                                        dh1, kHid, nullptr, false, 1)))
        return e;
    k_relu_mask<<<(unsigned)((n * kHid + 255) / 256), 256, 0, stream>>>(dh1, h1, n * kHid);
    if ((e = cudaGetLastError())) return e;
    // layer 1: dW1 = x^T dh1, db1 = colsum dh1
    if ((e = gemm<uint16_t, float>(stream, kIn, kHid, M, f, 1, kFeatStride, dh1, kHid, 1,
                                   grad + kOffW1, kHid, nullptr, false, splits)))
        return e;
    k_colsum<<<kHid, 256, 0, stream>>>(dh1, n, kHid, grad + kOffB1);
    return cudaGetLastError();
}

cudaError_t Predictor::adam(float lr) {
    ++steps;
    const float bc1 = 1.f - std::pow(0.9f, (float)steps);
    const float bc2 = 1.f - std::pow(0.999f, (float)steps);
    k_adam<<<(kParams + 255) / 256, 256, 0, stream>>>(master, w, grad, adam_m, adam_v, kParams, lr,
                                                       bc1, bc2);
    return cudaGetLastError();
}

cudaError_t abort_labels(const unsigned *tx_aborts, uint64_t first, uint64_t n, uint8_t *y,
                         cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    k_labels<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(tx_aborts, first, n, y);
    return cudaGetLastError();
}

cudaError_t partition(const float *p, uint64_t first, uint64_t n, float thr, uint32_t *order,
                      uint32_t *counts, float *sums, uint32_t *scratch, cudaStream_t st) {
    if (n == 0 || n > (1ull << 20)) return cudaErrorInvalidValue;
    const uint32_t nb = (uint32_t)((n + kPartBlock - 1) / kPartBlock);
    uint32_t *cnt = scratch;
    float *bsum = (float *)(scratch + nb);
    k_part_count<<<nb, kPartBlock, 0, st>>>(p, n, thr, cnt, bsum);
    k_part_scan<<<1, 32, 0, st>>>(cnt, bsum, nb, n, counts, sums);
    k_part_scatter<<<nb, kPartBlock, 0, st>>>(p, first, n, thr, cnt, counts, order);
    return cudaGetLastError();
}

}  // namespace sched
}  // namespace gcc
