// calib.cu -- the L2 atomic throughput a B200 sustains on the access pattern
// of the engine's CC metadata, as the denominator for the transaction
// kernel's measured atomic rate (the path is bound by dependent L2 round
// trips and atomics, not by HBM bandwidth, at every contention level).
//
// Pattern: one 64-bit word per row in a separate array (the lock / timestamp
// words, gcc_common.cuh), each atomic to a pseudo-random word. Modes:
//   GCC_CALIB_ADD  atomicAdd (2PL shared-lock increments, ticket counters)
//   GCC_CALIB_CAS  a load then an atomicCAS on the loaded value (2PL
//                  exclusive locks, OCC locks; a CAS that meets another
//                  thread's update fails and still counts as one atomic)
// Every thread issues `per_thread` atomics with up to 8 in flight (the
// transaction kernel has one per request lane in flight), over a resident
// grid of every SM. The array is at most the L2's size so that, as in the
// transaction kernel, the words stay in L2 after the first touch.
#include <cuda_runtime.h>
#include <algorithm>
#include "gcc_common.cuh"

namespace {

__global__ void __launch_bounds__(256) k_atomic_calib(unsigned long long *w, uint64_t mask,
                                                     uint32_t per_thread, int mode) {
    const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    unsigned long long acc = 0;
    for (uint32_t i = 0; i < per_thread; i += 8) {
        unsigned long long r[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const uint64_t a = gcc::splitmix64(t * 0x100000001ull + i + j) & mask;
            if (mode == GCC_CALIB_ADD) {
                r[j] = atomicAdd(w + a, 1ull);
            } else {
                // compare against the value the word holds for this thread's
                // turn: a plain load first, as a lock acquisition reads the
                // word before its CAS
                const unsigned long long old = __ldcg(w + a);
                r[j] = atomicCAS(w + a, old, old + 1ull);
            }
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) acc += r[j];
    }
    if (acc == 0x5eedull) w[0] = acc;  // keep the results live
}

}  // namespace

extern "C" int gcc_l2_atomic_rate(int32_t device, uint64_t words, int32_t mode,
                                  double *atomics_per_s) {
    cudaGetLastError();  // a stale error of an earlier call is not ours
    if (!atomics_per_s || (mode != GCC_CALIB_ADD && mode != GCC_CALIB_CAS)) return GCC_EINVAL;
    if (words < 1024 || (words & (words - 1)) || words > (1ull << 24)) return GCC_EINVAL;
    *atomics_per_s = 0;
    if (cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        return GCC_ENODEV;
    }
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
        cudaGetLastError();
        return GCC_ENODEV;
    }
    unsigned long long *w = nullptr;
    if (cudaMalloc(&w, words * 8) != cudaSuccess) {
        cudaGetLastError();
        return GCC_ENOMEM;
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    const int block = 256, grid = sms * 8;  // 2,048 threads per SM
    const uint32_t per_thread = 256;
    int rc = GCC_OK;
    float ms = 0.f;
    if (cudaMemset(w, 0, words * 8) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
        cudaEventCreate(&e1) != cudaSuccess) {
        rc = GCC_ECUDA;
    } else {
        // one warm-up pass brings the words into L2, then the timed pass
        k_atomic_calib<<<grid, block>>>(w, words - 1, per_thread, mode);
        cudaEventRecord(e0);
        k_atomic_calib<<<grid, block>>>(w, words - 1, per_thread, mode);
        cudaEventRecord(e1);
        if (cudaEventSynchronize(e1) != cudaSuccess || cudaGetLastError() != cudaSuccess)
            rc = GCC_ECUDA;
        else
            cudaEventElapsedTime(&ms, e0, e1);
    }
    if (rc == GCC_OK && ms > 0.f)
        *atomics_per_s = (double)grid * block * per_thread / (ms * 1e-3);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(w);
    cudaGetLastError();
    return rc;
}
