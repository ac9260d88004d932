// sched.cuh -- learned contention predictor of the scheduled executor.
//
// A small MLP estimates, for each transaction of a batch, the probability
// that it aborts at least once when the batch runs under plain ordering at
// full concurrency. The scheduler (engine.cu, gcc_sched_run) uses the
// estimates to defer predicted-conflicting transactions into a later
// sub-batch with fewer transactions in flight. The predictor changes no CC
// arithmetic and no commit rule; it only orders and groups transactions.
//
// Features of a transaction (66 values, u16, row stride 72):
//   [0, 64)  count sketch: requests whose key hashes (splitmix64) to each of
//            64 bins;
//   64       write requests;
//   65       hot-key hits, graded: the sum over requests of
//            floor(log2(1 + c)), c the key's counter in the device-side
//            frequency table (2^20 hashed counters, halved after every batch
//            and incremented by every request of the batch). A key seen once
//            in the last batches adds 1, one seen 65,535 times adds 16, so
//            the feature separates warm keys from the few very hot ones.
// The network reads feature / 16.
//
// Network: 66 -> 128 (ReLU) -> 128 (ReLU) -> 1 (sigmoid); BF16 weights and
// biases, FP32 activations and accumulation. Training keeps FP32 master
// weights with Adam and rounds them to BF16 after every step. The loss is
// the mean binary cross-entropy against labels "aborted at least once".
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "gcc_common.cuh"

namespace gcc {
namespace sched {

constexpr int kIn = 66;
constexpr int kFeatStride = 72;  // u16 per feature row (144 B, 16 B aligned)
constexpr int kSketch = 64;
constexpr int kHid = 128;
constexpr int kFreqBits = 20;
constexpr uint32_t kFreqSize = 1u << kFreqBits;
constexpr float kFeatScale = 1.0f / 16.0f;

// Flat parameter layout (master FP32, BF16 copy and gradients alike).
constexpr int kOffW1 = 0;                    // W1[i][u], i < 66, u < 128
constexpr int kOffB1 = kOffW1 + kIn * kHid;  // b1[u]
constexpr int kOffW2 = kOffB1 + kHid;        // W2[k][j]
constexpr int kOffB2 = kOffW2 + kHid * kHid; // b2[j]
constexpr int kOffW3 = kOffB2 + kHid;        // w3[j]
constexpr int kOffB3 = kOffW3 + kHid;        // b3
constexpr int kParams = kOffB3 + 1;          // 25,217

// floor(log2(1 + c)): a request's contribution to the hot-key feature.
GCC_HD uint32_t heat(uint32_t c) {
#ifdef __CUDA_ARCH__
    return c == 0xFFFFFFFFu ? 32u : 31u - (uint32_t)__clz((int)(c + 1u));
#else
    return c == 0xFFFFFFFFu ? 32u : 31u - (uint32_t)__builtin_clz(c + 1u);
#endif
}

// Key hashes of the sketch and of the frequency table.
GCC_HD uint32_t sketch_bin(uint32_t key) { return (uint32_t)(splitmix64(key) & 63u); }
GCC_HD uint32_t freq_slot(uint32_t key) {
    return (uint32_t)(splitmix64((uint64_t)key ^ 0x5EEDF00Dull) >> (64 - kFreqBits));
}

// Device buffers and launches of the predictor. All calls are asynchronous
// on `stream` and return the first CUDA error.
struct Predictor {
    int dev = 0;
    cudaStream_t stream = nullptr;
    uint64_t cap = 0;              // rows the activation buffers hold
    float *master = nullptr;       // FP32 weights (Adam)
    __nv_bfloat16 *w = nullptr;    // BF16 weights used by every pass
    float *grad = nullptr, *adam_m = nullptr, *adam_v = nullptr;
    float *h1 = nullptr, *h2 = nullptr, *dh1 = nullptr, *dh2 = nullptr;
    float *p = nullptr, *dz = nullptr, *loss = nullptr;
    uint8_t *labels = nullptr;
    uint16_t *feat = nullptr;
    uint32_t *freq = nullptr;
    uint64_t steps = 0;            // Adam steps taken

    ~Predictor();
    cudaError_t init(int device, cudaStream_t st, uint64_t rows, uint64_t seed);
    cudaError_t reserve(uint64_t rows);
    // Host <-> device FP32 master weights (the BF16 copy is refreshed).
    cudaError_t set_weights(const float *host);
    cudaError_t get_weights(float *host);
    // features of transactions first .. first + n - 1 into feat[0 .. n)
    cudaError_t features(const gcc_ycsb_tx *txs, uint64_t first, uint64_t n, uint16_t *out);
    // the same for variable-length transactions (CSR: requests
    // reqs[tx_off[t] .. tx_off[t+1]), up to 64)
    cudaError_t features_var(const uint32_t *tx_off, const gcc_ycsb_req *reqs, uint64_t first,
                             uint64_t n, uint16_t *out);
    // frequency table: halve every counter, then count the batch's requests
    cudaError_t observe(const gcc_ycsb_tx *txs, uint64_t first, uint64_t n);
    cudaError_t observe_var(const uint32_t *tx_off, const gcc_ycsb_req *reqs, uint64_t first,
                            uint64_t n);
    cudaError_t clear_freq();
    // 2PL lock plans (KParams::plan) of transactions first .. first + n - 1
    // into plan[first ..]: requests whose key counter is >= thr are locked
    // last, the hottest last of all
    cudaError_t lock_plan(const gcc_ycsb_tx *txs, uint64_t first, uint64_t n, uint32_t thr,
                          unsigned long long *plan);
    // p[0 .. n) = network(feat rows); activations stay in h1/h2
    cudaError_t forward(const uint16_t *f, uint64_t n, float *p_out);
    // gradient of the mean BCE over n rows into grad (and the loss summed
    // over the rows into *loss); labels are 0/1 bytes
    cudaError_t gradient(const uint16_t *f, const uint8_t *y, uint64_t n);
    // one Adam step on grad
    cudaError_t adam(float lr);
};

// Labels of a batch: y[i] = tx_aborts[first + i] > 0.
cudaError_t abort_labels(const unsigned *tx_aborts, uint64_t first, uint64_t n, uint8_t *y,
                         cudaStream_t st);

// Stable partition of positions 0 .. n-1 by p[i] > thr into
// order[0 .. n_low) (p <= thr, transaction order) then the rest; writes
// order entries first + i, and counts[0] = n_low, sums[0] = sum of p over the
// batch, sums[1] = sum of p over the deferred part. Needs n <= 2^20 and a
// scratch of (n + 1023) / 1024 * 3 u32.
cudaError_t partition(const float *p, uint64_t first, uint64_t n, float thr, uint32_t *order,
                      uint32_t *counts, float *sums, uint32_t *scratch, cudaStream_t st);

}  // namespace sched
}  // namespace gcc
