// noalloc.cu -- a 2PL no-wait run that allocates no device memory.
//
// Some callers cannot call cudaMalloc: code embedded in a process whose
// device memory belongs to another allocator (a framework's caching pool, a
// pre-sized arena in a real-time service), or that runs on a latency-bound
// thread where cudaMalloc's implicit device synchronisation is not
// acceptable. For them, gcc_run_tpl_nw_noalloc executes the YCSB
// transactions under 2PL no-wait with the caller's own device buffers for
// every input and output, and keeps its scratch memory (one lock word per
// row plus the run counters) in the file-scope device array below instead of
// allocating it.
//
// Limits and sharing:
//   * at most kNoAllocMaxRows rows (8 MiB of lock words); larger tables are
//     rejected with GCC_EINVAL;
//   * the array exists once per GPU that loads this library and stays
//     allocated until the process exits;
//   * every call on a device uses the same array and leaves its contents
//     behind; each call clears the lock words and counters it uses before
//     launching, so calls must not overlap on the GPU: two calls running at
//     the same time (e.g. on two streams) race on the array;
//   * the first call on each device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current, together with the
//     device's SM count and the kernel's occupancy; make that first call
//     before any stream capture on the device. The address belongs to the
//     device's primary context: after cudaDeviceReset on a device the
//     looked-up address is stale and this entry point must not be called on
//     that device again in the same process;
//   * the function returns only once its kernel has finished (also on an
//     error after the launch), so the caller may reuse or free its buffers
//     as soon as it returns.
#include <cuda_runtime.h>
#include <mutex>

#include "cc_kernel.cuh"

namespace {

constexpr uint64_t kNoAllocMaxRows = 1ull << 20;  // 1,048,576 rows
constexpr size_t kLockBytes = kNoAllocMaxRows * sizeof(unsigned long long);
constexpr size_t kCounterOffset = kLockBytes;  // 256-aligned (kLockBytes is)
constexpr size_t kScratchBytes = kCounterOffset + ((sizeof(gcc::Counters) + 255) / 256) * 256;

// Scratch of gcc_run_tpl_nw_noalloc: lock words, then the Counters block.
// Host code must not use this name as a pointer (it is a host-side stand-in,
// not a device address); it uses the address from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
constexpr int kG = 32, kBlock = 1024;  // one transaction per warp, 1024-thread CTAs

// What a call needs to know about a device, looked up once per device.
struct DeviceSetup {
    unsigned char *scratch = nullptr;  // device address of g_noalloc_scratch
    int grid_cap = 0;                  // resident CTAs: occupancy x SMs
};
std::mutex g_mu;
DeviceSetup g_setup[kMaxDevices];

// Set-up of device `dev` (current): the scratch array's device address, and
// the persistent grid the kernel fills. Done on the first call per device.
int device_setup(int dev, DeviceSetup *out) {
    if (dev < 0 || dev >= kMaxDevices) return GCC_ENODEV;
    std::lock_guard<std::mutex> lk(g_mu);
    DeviceSetup &d = g_setup[dev];
    if (!d.scratch) {
        int major = 0, sms = 0, occ = 0;
        if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
            cudaGetLastError();
            return GCC_ENODEV;
        }
        if (major < 10) return GCC_ENODEV;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                &occ, gcc::ycsb_kernel<gcc::S_TPL_NW, kG>, kBlock, 0) != cudaSuccess || occ <= 0) {
            cudaGetLastError();
            return GCC_ECUDA;
        }
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return GCC_ECUDA;
        }
        d.grid_cap = occ * sms;
        d.scratch = (unsigned char *)p;
    }
    *out = d;
    return GCC_OK;
}

}  // namespace

extern "C" int gcc_run_tpl_nw_noalloc(const gcc_ycsb_tx *txs, uint64_t n_tx, void *table,
                                      uint64_t rows, uint64_t *digests, uint32_t *tx_aborts,
                                      uint64_t write_seed, void *stream, uint64_t *committed,
                                      uint64_t *aborts) {
    cudaGetLastError();  // a stale error of an earlier call is not ours
    if (!txs || !table || !digests || !tx_aborts) return GCC_EINVAL;
    if (rows == 0 || rows > kNoAllocMaxRows) return GCC_EINVAL;
    if (n_tx == 0 || n_tx >= (1ull << 27)) return GCC_EINVAL;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return GCC_ENODEV;
    }
    DeviceSetup ds;
    int rc = device_setup(dev, &ds);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    gcc::Counters *ctr = (gcc::Counters *)(ds.scratch + kCounterOffset);
    unsigned long long *locks = (unsigned long long *)ds.scratch;
    // The array keeps the previous call's contents: clear what starts at
    // zero. A failure here happens before anything of ours is queued after
    // it, but an earlier memset may be queued: wait for the stream before
    // returning so that nothing of this call is still running.
    if (cudaMemsetAsync(locks, 0, rows * sizeof(unsigned long long), st) != cudaSuccess ||
        cudaMemsetAsync(ctr, 0, sizeof(gcc::Counters), st) != cudaSuccess) {
        cudaStreamSynchronize(st);
        cudaGetLastError();
        return GCC_ECUDA;
    }

    gcc::KParams p;
    memset(&p, 0, sizeof(p));
    p.txs = txs;
    p.n_tx = (uint32_t)n_tx;
    p.slot_ops = gcc::kMaxOps;
    p.batch_st = 0;
    p.batch_n = (uint32_t)n_tx;
    p.index_kind = GCC_INDEX_DIRECT;  // keys are row ids
    p.rows = rows;
    p.table = (uint8_t *)table;
    p.stride = gcc_row_stride(GCC_LAYOUT_U64X11);
    p.words = gcc_row_bytes(GCC_LAYOUT_U64X11) / 8;
    p.wslot = (p.words + 1) & ~1u;
    p.write_mode = GCC_WRITE_FIELD;
    p.write_seed = write_seed;
    p.meta = locks;
    p.digest = (unsigned long long *)digests;
    p.tx_aborts = tx_aborts;
    p.ctr = ctr;
    p.spin_limit_ns = 4000000000ull;
    p.backoff_ns = 512;
    // starvation control as gcc_run's default (starve_limit 0 -> 32): under
    // contention a transaction that keeps aborting pauses new admissions and
    // later retries under a token, which bounds retry cycles
    p.starve_limit = 32;

    const uint64_t want = (n_tx * kG + kBlock - 1) / kBlock;
    const int grid = (int)(want < (uint64_t)ds.grid_cap ? want : (uint64_t)ds.grid_cap);
    gcc::ycsb_kernel<gcc::S_TPL_NW, kG><<<grid, kBlock, 0, st>>>(p);
    const cudaError_t le = cudaGetLastError();
    unsigned long long host[2] = {0, 0};
    unsigned err = 0;
    bool ok = le == cudaSuccess &&
              cudaMemcpyAsync(host, &ctr->committed, 2 * sizeof(unsigned long long),
                              cudaMemcpyDeviceToHost, st) == cudaSuccess &&
              cudaMemcpyAsync(&err, &ctr->err, sizeof(unsigned), cudaMemcpyDeviceToHost, st) ==
                  cudaSuccess;
    // Wait for the stream on every path: the kernel may still be writing the
    // caller's table, digests and abort counts, and the shared scratch.
    ok = (cudaStreamSynchronize(st) == cudaSuccess) && ok;
    if (!ok) {
        cudaGetLastError();
        return GCC_ECUDA;
    }
    if (committed) *committed = host[0];
    if (aborts) *aborts = host[1];
    if (err) return (int)err;
    return host[0] == n_tx ? GCC_OK : GCC_ESTATE;
}
