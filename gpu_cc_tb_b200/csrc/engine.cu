// engine.cu -- host side of the C ABI: device memory layout, the batch loop,
// per-scheme metadata resets, GaccO/GPUTx ordering passes and result readout.
//
// Reference behaviour followed:
//   host driver / batch loop            benchmark_cpu/ycsb.cu:81-302
//   batching into ceil(tx/batch) runs    include/cc.cuh:29-35
//   per-batch metadata resets            twopl.cuh:431-435, to.cuh:316-321,
//                                        mvcc.cuh:351-376, silo.cuh:379-383,
//                                        tictoc.cuh:409-413
//   GaccO per-batch precompute           include/gacco.cuh:244-339
//   GPUTx ranking over all transactions  include/gputx.cuh:213-299
//   metrics + output line                include/runtime.cuh:169-214
#include <cuda_runtime.h>
#include <algorithm>
#include <chrono>
#include <cmath>
#include <map>
#include <cstdio>
#include <cstring>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "cc_launch.cuh"
#include "prep_kernels.cuh"
#include "sched.cuh"

using namespace gcc;

namespace {

struct SchemeName {
    const char *name;
    int id;
};
const SchemeName kSchemes[] = {
    {"tpl_nw", S_TPL_NW},       {"tpl_wd", S_TPL_WD},           {"to", S_TO},
    {"mvcc", S_MVCC},           {"silo", S_SILO},               {"tictoc", S_TICTOC},
    {"gacco", S_GACCO},         {"gputx", S_GPUTX},             {"slow_tpl_nw", S_SLOW_TPL_NW},
    {"slow_tpl_wd", S_SLOW_TPL_WD}, {"slow_to", S_SLOW_TO},     {"slow_mvcc", S_SLOW_MVCC},
    {"slow_silo", S_SLOW_SILO}, {"slow_tictoc", S_SLOW_TICTOC},
    // spellings found in the reference's result files / tpcc driver
    {"slowto", S_SLOW_TO},      {"slowmvcc", S_SLOW_MVCC},
};

// Grid that holds at most max_active transactions of G lanes in CTAs of
// `block` threads (0: no cap).
uint64_t active_grid(int32_t max_active, int G, int block) {
    if (max_active <= 0) return ~0ull;
    return std::max<uint64_t>(1, ((uint64_t)max_active * G + block - 1) / block);
}

// Latency percentile q (0..1) of a run's log-linear histogram in
// microseconds: the upper edge of the bucket that reaches the q-th
// transaction (buckets: 1 ns below 16 ns, then 16 linear steps per octave).
double hist_percentile_us(const Counters &hc, double q) {
    uint64_t total = 0;
    for (int i = 0; i < kHistBuckets; ++i) total += hc.hist[i];
    if (!total) return 0.0;
    auto edge = [](int b) -> double {
        if (b < 16) return (double)b + 1.0;
        const int lg = b / 16 + 3, sub = b % 16;
        return std::ldexp(16.0 + sub + 1.0, lg - 4);
    };
    const uint64_t target = (uint64_t)std::ceil(q * (double)total);
    uint64_t acc = 0;
    for (int i = 0; i < kHistBuckets; ++i) {
        acc += hc.hist[i];
        if (acc >= target) return edge(i) / 1000.0;
    }
    return edge(kHistBuckets - 1) / 1000.0;
}

// starve_limit of gcc_run_params -> kernel value (0: off)
uint32_t starve_param(int32_t v) { return v < 0 ? 0u : (v == 0 ? 32u : (uint32_t)v); }

bool is_slow(int s) { return s >= S_SLOW_TPL_NW; }
// Schemes whose CC metadata stays valid from one batch to the next, so that
// batches can share one launch (GCC_F_QUEUE): 2PL releases every lock,
// Silo / TicToc words only grow, TO timestamps keep growing when the
// counter is not reset. Not MVCC (its version store is indexed by batch
// position) nor the ordered schemes (per-batch ordering passes).
bool queue_scheme(int s) {
    return s == S_TPL_NW || s == S_TPL_WD || s == S_TO || s == S_SILO || s == S_TICTOC ||
           s == S_SLOW_TPL_NW || s == S_SLOW_TPL_WD || s == S_SLOW_TO || s == S_SLOW_SILO ||
           s == S_SLOW_TICTOC;
}
bool uses_ts(int s) { return s == S_TO || s == S_SLOW_TO || s == S_MVCC || s == S_SLOW_MVCC; }
bool is_mvcc(int s) { return s == S_MVCC || s == S_SLOW_MVCC; }

cudaError_t launch_scheme_kernel(int s, int G, int grid, int block, const KParams &p,
                                 cudaStream_t st) {
    switch (s) {
        case S_TPL_NW: case S_TPL_WD: case S_SLOW_TPL_NW: case S_SLOW_TPL_WD:
            return launch_family_tpl(s, G, grid, block, p, st);
        case S_TO: case S_SLOW_TO: return launch_family_to(s, G, grid, block, p, st);
        case S_MVCC: case S_SLOW_MVCC: return launch_family_mvcc(s, G, grid, block, p, st);
        case S_SILO: case S_SLOW_SILO: return launch_family_silo(s, G, grid, block, p, st);
        case S_TICTOC: case S_SLOW_TICTOC: return launch_family_tictoc(s, G, grid, block, p, st);
        default: return launch_family_ordered(s, G, grid, block, p, st);
    }
}
int scheme_occupancy(int s, int G, int block) {
    switch (s) {
        case S_TPL_NW: case S_TPL_WD: case S_SLOW_TPL_NW: case S_SLOW_TPL_WD:
            return occupancy_family_tpl(s, G, block);
        case S_TO: case S_SLOW_TO: return occupancy_family_to(s, G, block);
        case S_MVCC: case S_SLOW_MVCC: return occupancy_family_mvcc(s, G, block);
        case S_SILO: case S_SLOW_SILO: return occupancy_family_silo(s, G, block);
        case S_TICTOC: case S_SLOW_TICTOC: return occupancy_family_tictoc(s, G, block);
        default: return occupancy_family_ordered(s, G, block);
    }
}

inline unsigned grid1d(uint64_t n, unsigned block) {
    return (unsigned)((n + block - 1) / block);
}
int bits_for(uint64_t maxval) {  // bits to represent 0..maxval
    int b = 1;
    while (b < 32 && (1ull << b) <= maxval) ++b;
    return b;
}

}  // namespace

#define CK(call)                                   \
    do {                                           \
        cudaError_t e_ = (call);                   \
        if (e_ != cudaSuccess) {                   \
            last_cuda = e_;                        \
            return GCC_ECUDA;                      \
        }                                          \
    } while (0)

struct gcc_engine {
    int dev = 0;
    int sm_count = 0;
    int clock_khz = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t copy_in = nullptr, copy_out = nullptr;  // gcc_run_host transfers
    const gcc_ycsb_tx *host_src = nullptr;              // set during gcc_run_host
    uint64_t *host_dg = nullptr;
    cudaError_t last_cuda = cudaSuccess;
    gcc_table_desc desc{};
    uint32_t row_bytes = 0, stride = 0, words = 0, wslot = 0;
    uint64_t rows = 0;
    uint8_t *table = nullptr;
    // index
    unsigned long long *hash_slots = nullptr;
    uint64_t hash_bucket_mask = 0;
    unsigned long long *sorted = nullptr;
    // transactions
    gcc_ycsb_tx *txs = nullptr;
    uint64_t n_rec = 0, cap_rec = 0;  // 16-request records loaded / capacity
    uint64_t n_tx = 0, cap_tx = 0;    // transactions the per-tx outputs cover
    // per-row metadata
    unsigned long long *meta = nullptr;
    unsigned *latch = nullptr;
    unsigned *turn = nullptr;
    // per-tx outputs
    unsigned long long *digest = nullptr, *commit_hi = nullptr, *commit_lo = nullptr;
    unsigned *tx_aborts = nullptr;
    uint64_t *read_log = nullptr;
    uint64_t read_log_units = 0;
    // per-access scratch (units = positions)
    uint64_t *scratch = nullptr;
    uint64_t scratch_units = 0;
    unsigned long long *ver_ts = nullptr;
    unsigned *ver_prev = nullptr;
    uint64_t *ver_data = nullptr;
    uint64_t ver_units = 0;
    // ordering passes
    uint32_t *acc_key[2] = {nullptr, nullptr}, *acc_val[2] = {nullptr, nullptr};
    uint32_t *op_row = nullptr, *op_pos = nullptr, *order = nullptr, *tx_rank = nullptr;
    uint32_t *sort_counts = nullptr;
    uint64_t acc_cap = 0, counts_cap = 0, order_cap = 0;
    std::vector<uint32_t *> scan_tmp;
    std::vector<uint64_t> scan_tmp_n;
    Counters *ctr = nullptr;
    // variable-length transactions (CSR) and the batched executors
    uint32_t *tx_off_d = nullptr;
    gcc_ycsb_req *reqs_d = nullptr;
    uint64_t n_var = 0, var_ops = 0, cap_var = 0, cap_var_ops = 0;
    std::vector<uint32_t> tx_off_h;  // host copy of the offsets (batch classes)
    unsigned long long *queue_tail = nullptr;
    uint64_t *tail_h = nullptr;  // pinned: queue tail after each batch (GCC_F_QUEUE)
    uint64_t tail_cap = 0;
    unsigned long long *stamps = nullptr;  // device time stamps of batched runs
    uint64_t stamps_cap = 0;
    struct Arm {
        int wd, bs, div;     // grid = the full persistent grid / div
        uint32_t split;      // batch_size: at most this many transactions per
                             // launch inside a batch (0: the whole batch)
        uint64_t active;     // transactions in flight under this arm
        double ms_per_tx = 0;
        uint64_t runs = 0;
    };
    std::map<int, std::vector<Arm>> tuner;  // batch class -> candidate configs
    cudaGraphExec_t graph = nullptr;
    std::vector<uint64_t> graph_key;
    std::vector<int32_t> bstat_wd, bstat_bs;
    std::vector<double> bstat_ms;
    std::vector<uint64_t> bstat_active;
    std::vector<uint32_t> bstat_split;
    // timing
    std::vector<cudaEvent_t> events;
    double last_kernel_ms = 0;
    uint64_t last_launches = 0;
    uint64_t kernel_launches = 0;
    bool have_run = false;

    ~gcc_engine();
    int fail_cuda(cudaError_t e) {
        last_cuda = e;
        return GCC_ECUDA;
    }
    template <class T>
    int alloc(T **p, size_t bytes) {
        if (*p) {
            cudaFree(*p);
            *p = nullptr;
        }
        if (bytes == 0) bytes = 16;
        cudaError_t e = cudaMalloc((void **)p, bytes);
        if (e != cudaSuccess) {
            *p = nullptr;
            last_cuda = e;
            cudaGetLastError();
            return e == cudaErrorMemoryAllocation ? GCC_ENOMEM : GCC_ECUDA;
        }
        return GCC_OK;
    }
    int ensure_events(size_t n) {
        while (events.size() < n) {
            cudaEvent_t ev;
            CK(cudaEventCreate(&ev));
            events.push_back(ev);
        }
        return GCC_OK;
    }
    KParams base_params() const;
    int radix_sort(uint64_t n, int bits, uint32_t **keys, uint32_t **vals);
    int scan(const uint32_t *in, uint32_t *out, uint64_t n, bool inclusive, int level = 0);
    int ensure_access(uint64_t n_acc);
    int order_pass(const KParams &p, uint64_t n_pos, int sched_bits);
    int gputx_rank(const KParams &p0);
};

gcc_engine::~gcc_engine() {
    if (dev >= 0) cudaSetDevice(dev);
    void *bufs[] = {table, hash_slots, sorted, txs, meta, latch, turn, digest, commit_hi,
                    commit_lo, tx_aborts, read_log, scratch, ver_ts, ver_prev, ver_data,
                    acc_key[0], acc_key[1], acc_val[0], acc_val[1], op_row, op_pos, order,
                    tx_rank, sort_counts, ctr, tx_off_d, reqs_d, queue_tail, stamps};
    for (void *b : bufs)
        if (b) cudaFree(b);
    for (uint32_t *t : scan_tmp)
        if (t) cudaFree(t);
    for (cudaEvent_t ev : events) cudaEventDestroy(ev);
    if (tail_h) cudaFreeHost(tail_h);
    if (graph) cudaGraphExecDestroy(graph);
    if (copy_in) cudaStreamDestroy(copy_in);
    if (copy_out) cudaStreamDestroy(copy_out);
    if (stream) cudaStreamDestroy(stream);
}

KParams gcc_engine::base_params() const {
    KParams p;
    memset(&p, 0, sizeof(p));
    p.txs = txs;
    p.n_tx = (uint32_t)n_tx;
    p.slot_ops = kMaxOps;
    p.index_kind = desc.index_kind;
    p.hash_slots = hash_slots;
    p.hash_bucket_mask = hash_bucket_mask;
    p.sorted = sorted;
    p.sorted_len = (uint32_t)rows;
    p.rows = rows;
    p.table = table;
    p.stride = stride;
    p.words = words;
    p.wslot = wslot;
    p.meta = meta;
    p.latch = latch;
    p.turn = turn;
    p.digest = digest;
    p.commit_hi = commit_hi;
    p.commit_lo = commit_lo;
    p.tx_aborts = tx_aborts;
    p.ctr = ctr;
    p.spin_limit_ns = 4000000000ull;
    return p;
}

// Multi-level exclusive/inclusive scan of u32.
int gcc_engine::scan(const uint32_t *in, uint32_t *out, uint64_t n, bool inclusive, int level) {
    if (n == 0) return GCC_OK;
    uint64_t nb = (n + kScanTile - 1) / kScanTile;
    if (nb == 1) {
        k_scan_tile<<<1, kScanThreads, 0, stream>>>(in, out, n, nullptr, inclusive ? 1 : 0);
        CK(cudaGetLastError());
        kernel_launches += 1;
        return GCC_OK;
    }
    while ((int)scan_tmp.size() <= level) {
        scan_tmp.push_back(nullptr);
        scan_tmp_n.push_back(0);
    }
    if (scan_tmp_n[level] < nb) {
        int rc = alloc(&scan_tmp[level], nb * sizeof(uint32_t));
        if (rc) return rc;
        scan_tmp_n[level] = nb;
    }
    uint32_t *sums = scan_tmp[level];
    k_scan_tile<<<(unsigned)nb, kScanThreads, 0, stream>>>(in, out, n, sums, inclusive ? 1 : 0);
    CK(cudaGetLastError());
    kernel_launches += 1;
    int rc = scan(sums, sums, nb, false, level + 1);
    if (rc) return rc;
    k_scan_add<<<(unsigned)nb, kScanThreads, 0, stream>>>(out, n, sums);
    CK(cudaGetLastError());
    kernel_launches += 1;
    return GCC_OK;
}

// Stable LSD radix sort of (keys, vals) over the low `bits` bits; the sorted
// pair ends in *keys / *vals (buffers may be swapped with the alternates).
int gcc_engine::radix_sort(uint64_t n, int bits, uint32_t **keys, uint32_t **vals) {
    if (n == 0) return GCC_OK;
    uint32_t nblocks = (uint32_t)((n + kSortTile - 1) / kSortTile);
    uint64_t ncounts = (uint64_t)nblocks * kRadix;
    if (counts_cap < ncounts) {
        int rc = alloc(&sort_counts, ncounts * sizeof(uint32_t));
        if (rc) return rc;
        counts_cap = ncounts;
    }
    uint32_t *ki = *keys, *vi = *vals;
    uint32_t *ko = (ki == acc_key[0]) ? acc_key[1] : acc_key[0];
    uint32_t *vo = (vi == acc_val[0]) ? acc_val[1] : acc_val[0];
    for (int shift = 0; shift < bits; shift += 8) {
        k_sort_hist<<<nblocks, kSortThreads, 0, stream>>>(ki, n, shift, sort_counts, nblocks);
        CK(cudaGetLastError());
        int rc = scan(sort_counts, sort_counts, ncounts, false);
        if (rc) return rc;
        k_sort_scatter<<<nblocks, kSortThreads, 0, stream>>>(ki, vi, n, shift, sort_counts,
                                                              nblocks, ko, vo);
        CK(cudaGetLastError());
        kernel_launches += 2;
        std::swap(ki, ko);
        std::swap(vi, vo);
    }
    *keys = ki;
    *vals = vi;
    return GCC_OK;
}

int gcc_engine::ensure_access(uint64_t n_acc) {
    if (acc_cap >= n_acc) return GCC_OK;
    int rc;
    for (int j = 0; j < 2; ++j) {
        if ((rc = alloc(&acc_key[j], n_acc * 4))) return rc;
        if ((rc = alloc(&acc_val[j], n_acc * 4))) return rc;
    }
    if ((rc = alloc(&op_row, n_acc * 4))) return rc;
    if ((rc = alloc(&op_pos, n_acc * 4))) return rc;
    acc_cap = n_acc;
    return GCC_OK;
}

// Access list of positions [p.batch_st, p.batch_st + n_pos) in p.order order:
// stable sort by row, then per-access positions and each row's first turn.
int gcc_engine::order_pass(const KParams &p, uint64_t n_pos, int) {
    uint64_t n_acc = n_pos * kMaxOps;
    int rc = ensure_access(n_acc);
    if (rc) return rc;
    int rbits = bits_for(rows);  // rows itself is the padding key
    uint32_t invalid = (uint32_t)rows;
    if (rbits > 32) return GCC_EINVAL;
    k_access_build<<<grid1d(n_acc, 256), 256, 0, stream>>>(p, n_pos, invalid, acc_key[0],
                                                           acc_val[0], op_row);
    CK(cudaGetLastError());
    kernel_launches += 1;
    uint32_t *k = acc_key[0], *v = acc_val[0];
    if ((rc = radix_sort(n_acc, rbits, &k, &v))) return rc;
    k_access_positions<<<grid1d(n_acc, 256), 256, 0, stream>>>(k, v, n_acc, invalid, op_pos,
                                                                turn);
    CK(cudaGetLastError());
    kernel_launches += 1;
    return GCC_OK;
}

// GPUTx ranking (gputx.cuh:213-299, src/gputx.cu:5-38) over all transactions,
// leaving the (rank, tx) execution order in `order`.
int gcc_engine::gputx_rank(const KParams &p0) {
    uint64_t n_acc = n_tx * kMaxOps;
    int rc = ensure_access(n_acc);
    if (rc) return rc;
    if (order_cap < n_tx) {
        if ((rc = alloc(&order, n_tx * 4))) return rc;
        if ((rc = alloc(&tx_rank, n_tx * 4))) return rc;
        order_cap = n_tx;
    }
    KParams p = p0;
    p.order = nullptr;
    p.batch_st = 0;
    uint32_t invalid = (uint32_t)rows;
    int rbits = bits_for(rows);
    k_access_build<<<grid1d(n_acc, 256), 256, 0, stream>>>(p, n_tx, invalid, acc_key[0],
                                                           acc_val[0], op_row);
    CK(cudaGetLastError());
    uint32_t *k = acc_key[0], *v = acc_val[0];
    if ((rc = radix_sort(n_acc, rbits, &k, &v))) return rc;
    // flags -> inclusive scan -> per-row base -> per-tx max rank
    uint32_t *f = (k == acc_key[0]) ? acc_key[1] : acc_key[0];
    uint32_t *S = op_pos;  // free until the second ordering pass
    k_rank_flags<<<grid1d(n_acc, 256), 256, 0, stream>>>(k, v, n_acc, invalid, f);
    CK(cudaGetLastError());
    if ((rc = scan(f, S, n_acc, true))) return rc;
    k_rank_segbase<<<grid1d(n_acc, 256), 256, 0, stream>>>(k, S, n_acc, invalid, turn);
    CK(cudaGetLastError());
    CK(cudaMemsetAsync(tx_rank, 0, n_tx * 4, stream));
    k_rank_tx<<<grid1d(n_acc, 256), 256, 0, stream>>>(k, v, S, n_acc, invalid, turn, tx_rank,
                                                       &ctr->max_rank);
    CK(cudaGetLastError());
    kernel_launches += 4;
    // stable sort of tx ids by rank: ranks < n_tx
    uint32_t *rk = (k == acc_key[0]) ? acc_key[1] : acc_key[0];
    uint32_t *rv = (v == acc_val[0]) ? acc_val[1] : acc_val[0];
    CK(cudaMemcpyAsync(rk, tx_rank, n_tx * 4, cudaMemcpyDeviceToDevice, stream));
    k_iota<<<grid1d(n_tx, 256), 256, 0, stream>>>(rv, n_tx);
    CK(cudaGetLastError());
    kernel_launches += 1;
    if ((rc = radix_sort(n_tx, bits_for(n_tx), &rk, &rv))) return rc;
    CK(cudaMemcpyAsync(order, rv, n_tx * 4, cudaMemcpyDeviceToDevice, stream));
    return GCC_OK;
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

const char *gcc_version(void) { return "gpu_cc_tb_b200 0.1 (sm_100a)"; }

const char *gcc_strerror(int status) {
    switch (status) {
        case GCC_OK: return "ok";
        case GCC_EINVAL: return "invalid argument";
        case GCC_ENOMEM: return "out of memory";
        case GCC_ECUDA: return "CUDA runtime error";
        case GCC_ETIMEOUT: return "bounded device wait timed out";
        case GCC_EFORMAT: return "malformed transaction record";
        case GCC_EKEY: return "request key not in index";
        case GCC_EOVERFLOW: return "timestamp space exhausted";
        case GCC_ESTATE: return "call out of order";
        case GCC_ENODEV: return "no usable CUDA device";
        default: return "unknown status";
    }
}

int gcc_scheme_id(const char *name) {
    if (!name) return GCC_EINVAL;
    for (const SchemeName &s : kSchemes)
        if (strcmp(s.name, name) == 0) return s.id;
    return GCC_EINVAL;
}

uint32_t gcc_row_bytes(int32_t layout) { return layout == GCC_LAYOUT_REF104 ? 104u : 88u; }
uint32_t gcc_row_stride(int32_t layout) { return layout == GCC_LAYOUT_REF104 ? 112u : 96u; }

int gcc_create(const gcc_table_desc *d, gcc_engine **out) {
    cudaGetLastError();  // a stale error of an earlier call is not ours
    if (!d || !out) return GCC_EINVAL;
    *out = nullptr;
    if (d->rows == 0 || d->rows >= 0xFFFFFFFFull) return GCC_EINVAL;
    if (d->layout != GCC_LAYOUT_U64X11 && d->layout != GCC_LAYOUT_REF104) return GCC_EINVAL;
    if (d->index_kind < GCC_INDEX_HASH || d->index_kind > GCC_INDEX_DIRECT) return GCC_EINVAL;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= d->device || d->device < 0) {
        cudaGetLastError();
        return GCC_ENODEV;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, d->device) != cudaSuccess) return GCC_ENODEV;
    if (prop.major < 10) return GCC_ENODEV;  // built for sm_100a only
    gcc_engine *e = new gcc_engine();
    e->dev = d->device;
    e->desc = *d;
    if (e->desc.max_batch <= 0) e->desc.max_batch = 65536;
    e->sm_count = prop.multiProcessorCount;
    int clk = 0;
    cudaDeviceGetAttribute(&clk, cudaDevAttrClockRate, d->device);
    e->clock_khz = clk > 0 ? clk : 1965000;
    e->rows = d->rows;
    e->row_bytes = gcc_row_bytes(d->layout);
    e->stride = gcc_row_stride(d->layout);
    e->words = e->row_bytes / 8;
    e->wslot = (e->words + 1) & ~1u;
    int rc = GCC_OK;
    auto bail = [&](int r) {
        delete e;
        return r;
    };
    if (cudaSetDevice(e->dev) != cudaSuccess) return bail(GCC_ENODEV);
    if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(GCC_ECUDA);
    if ((rc = e->alloc(&e->table, e->rows * e->stride))) return bail(rc);
    if ((rc = e->alloc(&e->meta, e->rows * 8))) return bail(rc);
    if ((rc = e->alloc(&e->turn, e->rows * 4))) return bail(rc);
    if ((rc = e->alloc(&e->ctr, sizeof(Counters)))) return bail(rc);
    if (cudaMemsetAsync(e->ctr, 0, sizeof(Counters), e->stream) != cudaSuccess) return bail(GCC_ECUDA);
    k_fill_table<<<grid1d(e->rows, 256), 256, 0, e->stream>>>(e->table, e->rows, e->stride,
                                                              e->words, d->layout, d->fill_seed);
    if (cudaGetLastError() != cudaSuccess) return bail(GCC_ECUDA);
    if (d->index_kind == GCC_INDEX_HASH) {
        uint64_t nb = 1;
        while (nb * 4 < 2 * e->rows) nb <<= 1;  // load factor <= 1/2
        e->hash_bucket_mask = nb - 1;
        if ((rc = e->alloc(&e->hash_slots, nb * 4 * 8))) return bail(rc);
        cudaMemsetAsync(e->hash_slots, 0xFF, nb * 4 * 8, e->stream);
        k_hash_insert<<<grid1d(e->rows, 256), 256, 0, e->stream>>>(
            e->table, e->rows, e->stride, e->hash_slots, e->hash_bucket_mask, &e->ctr->err);
        if (cudaGetLastError() != cudaSuccess) return bail(GCC_ECUDA);
    } else if (d->index_kind == GCC_INDEX_SORTED) {
        if ((rc = e->ensure_access(e->rows))) return bail(rc);
        k_sorted_entries<<<grid1d(e->rows, 256), 256, 0, e->stream>>>(
            e->table, e->rows, e->stride, e->acc_key[0], e->acc_val[0]);
        uint32_t *k = e->acc_key[0], *v = e->acc_val[0];
        if ((rc = e->radix_sort(e->rows, 32, &k, &v))) return bail(rc);
        if ((rc = e->alloc(&e->sorted, e->rows * 8))) return bail(rc);
        k_pack_sorted<<<grid1d(e->rows, 256), 256, 0, e->stream>>>(k, v, e->rows, e->sorted);
        if (cudaGetLastError() != cudaSuccess) return bail(GCC_ECUDA);
    }
    unsigned err = 0;
    if (cudaMemcpyAsync(&err, &e->ctr->err, 4, cudaMemcpyDeviceToHost, e->stream) != cudaSuccess ||
        cudaStreamSynchronize(e->stream) != cudaSuccess)
        return bail(GCC_ECUDA);
    if (err) return bail((int)err);
    *out = e;
    return GCC_OK;
}

void gcc_destroy(gcc_engine *e) { delete e; }

}  // extern "C"

// Device buffers for n_tx 16-request records and their per-tx outputs.
static int reserve_records(gcc_engine *e, uint64_t n_tx) {
    int rc;
    if (e->cap_rec < n_tx) {
        if ((rc = e->alloc(&e->txs, n_tx * sizeof(gcc_ycsb_tx)))) return rc;
        e->cap_rec = n_tx;
    }
    if (e->cap_tx < n_tx) {
        if ((rc = e->alloc(&e->digest, n_tx * 8))) return rc;
        if ((rc = e->alloc(&e->commit_hi, n_tx * 8))) return rc;
        if ((rc = e->alloc(&e->commit_lo, n_tx * 8))) return rc;
        if ((rc = e->alloc(&e->tx_aborts, n_tx * 4))) return rc;
        e->cap_tx = n_tx;
    }
    return GCC_OK;
}

extern "C" {

int gcc_load_txs(gcc_engine *e, const gcc_ycsb_tx *txs, uint64_t n_tx) {
    cudaGetLastError();  // a stale error of an earlier call is not ours
    if (!e || (!txs && n_tx)) return GCC_EINVAL;
    if (n_tx >= (1ull << 27)) return GCC_EINVAL;  // access ids must fit 31 bits
    cudaSetDevice(e->dev);
    int rc;
    if (e->cap_rec < n_tx) {
        if ((rc = e->alloc(&e->txs, n_tx * sizeof(gcc_ycsb_tx)))) return rc;
        e->cap_rec = n_tx;
    }
    if (e->cap_tx < n_tx) {
        if ((rc = e->alloc(&e->digest, n_tx * 8))) return rc;
        if ((rc = e->alloc(&e->commit_hi, n_tx * 8))) return rc;
        if ((rc = e->alloc(&e->commit_lo, n_tx * 8))) return rc;
        if ((rc = e->alloc(&e->tx_aborts, n_tx * 4))) return rc;
        e->cap_tx = n_tx;
    }
    e->n_tx = n_tx;
    e->n_rec = n_tx;
    e->have_run = false;
    if (n_tx) {
        cudaError_t ce = cudaMemcpyAsync(e->txs, txs, n_tx * sizeof(gcc_ycsb_tx),
                                         cudaMemcpyHostToDevice, e->stream);
        if (ce != cudaSuccess) return e->fail_cuda(ce);
    }
    return GCC_OK;
}

}  // extern "C"

// Runs with GCC_F_EXT_OPS: not under MVCC (versions hold whole rows written
// blindly), only on the u64 field layout with field writes.
static bool ext_ops_allowed(const gcc_engine *e, int s, const gcc_run_params *rp) {
    if (!(rp->flags & GCC_F_EXT_OPS)) return true;
    return !is_mvcc(s) && e->desc.layout == GCC_LAYOUT_U64X11 && rp->write_mode == GCC_WRITE_FIELD;
}

extern "C" {

int gcc_run(gcc_engine *e, const gcc_run_params *rp, gcc_result *out) {
    cudaGetLastError();  // a stale error of an earlier call is not ours
    if (!e || !rp || !out) return GCC_EINVAL;
    memset(out, 0, sizeof(*out));
    const int s = gcc_scheme_id(rp->cc_scheme);
    if (s < 0) return GCC_EINVAL;
    // knob ranges of benchmark_cpu/ycsb.cu:97-98 (block_size 0 would divide
    // by zero there, :260-270)
    if (rp->warp_density < 0 || rp->warp_density > 5) return GCC_EINVAL;
    if (rp->block_size < 1 || rp->block_size > 32) return GCC_EINVAL;
    if (rp->batch_size < 1) return GCC_EINVAL;
    if (rp->write_mode != GCC_WRITE_FIELD && rp->write_mode != GCC_WRITE_ROWCOPY) return GCC_EINVAL;
    if (rp->flags & GCC_F_EXT_OPS) return GCC_EINVAL;  // variable-length runs only
    if (!e->txs || e->n_rec == 0) return GCC_ESTATE;
    cudaSetDevice(e->dev);
    e->n_tx = e->n_rec;  // outputs of this run cover the records
    const int G = 1 << rp->warp_density;
    const int block = rp->block_size * 32;
    const bool gputx = s == S_GPUTX;
    const bool ordered = s == S_GACCO || gputx;
    const uint64_t batch = gputx ? e->n_tx : std::min<uint64_t>((uint64_t)rp->batch_size, e->n_tx);
    const uint64_t nbatches = (e->n_tx + batch - 1) / batch;
    const bool rowcopy = rp->write_mode == GCC_WRITE_ROWCOPY;
    const bool want_log = (rp->flags & GCC_F_READ_LOG) != 0;
    // GCC_F_QUEUE: one persistent launch drains every batch in order
    const bool queue = (rp->flags & GCC_F_QUEUE) != 0;
    if (queue && (!queue_scheme(s) || rowcopy)) return GCC_EINVAL;
    const uint64_t nlaunch = queue ? 1 : nbatches;
    int rc;

    // lazily sized per-run buffers
    if (rowcopy && e->scratch_units < batch) {
        if ((rc = e->alloc(&e->scratch, batch * kMaxOps * e->wslot * 8))) return rc;
        e->scratch_units = batch;
    }
    if (want_log && e->read_log_units < e->n_tx) {
        if ((rc = e->alloc(&e->read_log, e->n_tx * kMaxOps * e->wslot * 8))) return rc;
        e->read_log_units = e->n_tx;
    }
    if (is_mvcc(s) && e->ver_units < batch) {
        if ((rc = e->alloc(&e->ver_ts, batch * kMaxOps * 8))) return rc;
        if ((rc = e->alloc(&e->ver_prev, batch * kMaxOps * 4))) return rc;
        if ((rc = e->alloc(&e->ver_data, batch * kMaxOps * e->wslot * 8))) return rc;
        e->ver_units = batch;
    }
    if (is_slow(s) && !e->latch) {
        if ((rc = e->alloc(&e->latch, e->rows * 4))) return rc;
        cudaError_t ce = cudaMemsetAsync(e->latch, 0, e->rows * 4, e->stream);
        if (ce != cudaSuccess) return e->fail_cuda(ce);
    }
    if (want_log) {
        cudaError_t ce = cudaMemsetAsync(e->read_log, 0, e->n_tx * kMaxOps * e->wslot * 8, e->stream);
        if (ce != cudaSuccess) return e->fail_cuda(ce);
    }

    int occ = scheme_occupancy(s, G, block);
    if (occ <= 0) return GCC_EINVAL;  // block too large for this kernel
    if (rp->max_active < 0 || rp->starve_limit < -1 || rp->ordered_after < 0) return GCC_EINVAL;
    const uint64_t max_grid = std::min<uint64_t>((uint64_t)occ * e->sm_count,
                                                 active_grid(rp->max_active, G, block));

    KParams p = e->base_params();
    p.write_mode = rp->write_mode;
    p.write_seed = rp->write_seed;
    p.flags = rp->flags;
    p.spin_limit_ns = rp->spin_limit_ns ? rp->spin_limit_ns : 4000000000ull;
    p.wait_die = (s == S_TPL_WD || s == S_SLOW_TPL_WD) ? 1u : 0u;
    if (rp->backoff_ns < -1 || rp->backoff_ns > 100000) return GCC_EINVAL;
    p.backoff_ns = rp->backoff_ns < 0 ? 0u : (rp->backoff_ns == 0 ? 512u : (uint32_t)rp->backoff_ns);
    p.starve_limit = starve_param(rp->starve_limit);
    p.ordered_from = rp->ordered_after > 0 ? (uint32_t)rp->ordered_after + 1u : 0u;
    p.scratch = rowcopy ? e->scratch : nullptr;
    p.read_log = want_log ? e->read_log : nullptr;
    p.ver_ts = e->ver_ts;
    p.ver_prev = e->ver_prev;
    p.ver_data = e->ver_data;

    const bool streamed = e->host_src != nullptr;
    const uint64_t ev_copy = 3 * nbatches + 4;  // then nbatches copy-in, nbatches kernel-done
    if ((rc = e->ensure_events(3 * nbatches + 4 + (streamed ? 2 * nbatches : 0)))) return rc;
    cudaEvent_t ev_start = e->events[0], ev_pre0 = e->events[1], ev_stop = e->events[2];
    const uint64_t launches0 = e->kernel_launches;
    if (queue && streamed) {
        // the device queue's tail, and the pinned host values the copy
        // stream writes into it after each batch's records
        if (!e->queue_tail && (rc = e->alloc(&e->queue_tail, 8))) return rc;
        if (e->tail_cap < nbatches) {
            if (e->tail_h) cudaFreeHost(e->tail_h);
            e->tail_h = nullptr;
            e->tail_cap = 0;
            cudaError_t he = cudaHostAlloc((void **)&e->tail_h, nbatches * 8, cudaHostAllocDefault);
            if (he != cudaSuccess) {
                e->tail_h = nullptr;
                cudaGetLastError();
                return GCC_ENOMEM;
            }
            e->tail_cap = nbatches;
        }
        for (uint64_t b = 0; b < nbatches; ++b)
            e->tail_h[b] = std::min<uint64_t>((b + 1) * batch, e->n_tx);
    }

    cudaStream_t st = e->stream;
    cudaError_t ce;
#define CKR(call)                             \
    do {                                      \
        ce = (call);                          \
        if (ce != cudaSuccess) return e->fail_cuda(ce); \
    } while (0)
    CKR(cudaMemsetAsync(e->ctr, 0, sizeof(Counters), st));
    // (before ev_start: the copy stream's tail updates come after this)
    if (queue && streamed) CKR(cudaMemsetAsync(e->queue_tail, 0, 8, st));
    CKR(cudaEventRecord(ev_start, st));
    if (streamed) {
        // host records stream in batch by batch on their own stream; each
        // batch waits only for its own records (gcc_run_host); with the
        // device queue, each copy is followed by the queue tail's advance
        // past that batch
        if (!e->copy_in) CKR(cudaStreamCreateWithFlags(&e->copy_in, cudaStreamNonBlocking));
        if (!e->copy_out) CKR(cudaStreamCreateWithFlags(&e->copy_out, cudaStreamNonBlocking));
        CKR(cudaStreamWaitEvent(e->copy_in, ev_start, 0));
        for (uint64_t b = 0; b < nbatches; ++b) {
            const uint64_t bst = b * batch, bn = std::min<uint64_t>(batch, e->n_tx - bst);
            CKR(cudaMemcpyAsync(e->txs + bst, e->host_src + bst, bn * sizeof(gcc_ycsb_tx),
                                cudaMemcpyHostToDevice, e->copy_in));
            if (queue)
                CKR(cudaMemcpyAsync(e->queue_tail, e->tail_h + b, 8, cudaMemcpyHostToDevice,
                                    e->copy_in));
            CKR(cudaEventRecord(e->events[ev_copy + b], e->copy_in));
        }
    }
    // GPUTx ranks every transaction once, before the batches (Init0).
    if (gputx) {
        if (streamed) CKR(cudaStreamWaitEvent(st, e->events[ev_copy + nbatches - 1], 0));
        if ((rc = e->gputx_rank(p))) return rc;
        p.order = e->order;
    }
    CKR(cudaEventRecord(ev_pre0, st));
    for (uint64_t b = 0; b < nlaunch; ++b) {
        cudaEvent_t e0 = e->events[3 + 3 * b], e1 = e->events[4 + 3 * b], e2 = e->events[5 + 3 * b];
        const uint64_t bst = b * batch;
        // queue: the launch covers every position; batches are admitted
        // through the queue tail (streamed) or all at once
        const uint64_t bn = queue ? e->n_tx : std::min<uint64_t>(batch, e->n_tx - bst);
        p.batch_st = (uint32_t)bst;
        p.batch_n = (uint32_t)bn;
        p.queue_tail = (queue && streamed) ? e->queue_tail : nullptr;
        CKR(cudaEventRecord(e0, st));
        if (streamed && !queue) CKR(cudaStreamWaitEvent(st, e->events[ev_copy + b], 0));
        // per-batch metadata reset (the reference memsets the whole table).
        // 2PL lock words are all zero again once a batch has committed every
        // transaction (each lock taken is released), so for 2PL the memset
        // of later batches would rewrite zeros with zeros and is skipped:
        // the state is the reset state either way.
        const bool tpl2 = s == S_TPL_NW || s == S_TPL_WD || s == S_SLOW_TPL_NW || s == S_SLOW_TPL_WD;
        const bool keep = tpl2 || ((rp->flags & GCC_F_NO_RESET) &&
                                   (s == S_SILO || s == S_TICTOC || s == S_SLOW_SILO ||
                                    s == S_SLOW_TICTOC));
        if (!ordered && !(keep && b > 0)) CKR(cudaMemsetAsync(e->meta, 0, e->rows * 8, st));
        if (is_mvcc(s)) CKR(cudaMemsetAsync(e->turn, 0xFF, e->rows * 4, st));
        k_batch_prep<<<1, 32, 0, st>>>(e->ctr, uses_ts(s) ? 1 : 0);
        CKR(cudaGetLastError());
        e->kernel_launches += 1;
        if (s == S_GACCO) {
            if ((rc = e->order_pass(p, bn, 0))) return rc;
            p.op_row = e->op_row;
            p.op_pos = e->op_pos;
        } else if (gputx) {
            // second pass: accesses in (rank, tx) order
            if ((rc = e->order_pass(p, bn, 0))) return rc;
            p.op_row = e->op_row;
            p.op_pos = e->op_pos;
        }
        CKR(cudaEventRecord(e1, st));
        uint64_t want = (bn * (uint64_t)G + block - 1) / block;
        int grid = (int)std::max<uint64_t>(1, std::min<uint64_t>(want, max_grid));
        CKR(launch_scheme_kernel(s, G, grid, block, p, st));
        e->kernel_launches += 1;
        CKR(cudaEventRecord(e2, st));
        if (streamed && e->host_dg) {
            // the batch's read digests go back while later batches run
            // (queue: all of them after the one launch)
            CKR(cudaStreamWaitEvent(e->copy_out, e2, 0));
            CKR(cudaMemcpyAsync(e->host_dg + bst, e->digest + bst, bn * 8, cudaMemcpyDeviceToHost,
                                e->copy_out));
        }
    }
    CKR(cudaEventRecord(ev_stop, st));
    CKR(cudaStreamSynchronize(st));
    if (streamed) {
        CKR(cudaStreamSynchronize(e->copy_in));
        CKR(cudaStreamSynchronize(e->copy_out));
    }
#undef CKR

    Counters hc;
    ce = cudaMemcpy(&hc, e->ctr, sizeof(Counters), cudaMemcpyDeviceToHost);
    if (ce != cudaSuccess) return e->fail_cuda(ce);
    e->have_run = true;
    float ms = 0;
    double pre_ms = 0, proc_ms = 0;
    cudaEventElapsedTime(&ms, ev_start, ev_pre0);
    pre_ms += ms;
    for (uint64_t b = 0; b < nlaunch; ++b) {
        cudaEventElapsedTime(&ms, e->events[3 + 3 * b], e->events[4 + 3 * b]);
        pre_ms += ms;
        cudaEventElapsedTime(&ms, e->events[4 + 3 * b], e->events[5 + 3 * b]);
        proc_ms += ms;
    }
    cudaEventElapsedTime(&ms, ev_start, ev_stop);
    double tot_ms = ms;
    e->last_kernel_ms = proc_ms;
    e->last_launches = nlaunch;

    out->committed = hc.committed;
    out->aborts = hc.aborts;
    out->pre_s = pre_ms / 1000.0;
    out->proc_s = proc_ms / 1000.0;
    out->tot_s = tot_ms / 1000.0;
    out->tx_per_s = tot_ms > 0 ? (double)hc.committed * 1000.0 / tot_ms : 0.0;
    const double inv = 1.0 / ((double)e->n_tx * (double)e->clock_khz);
    out->ts_d = hc.ts_cycles * inv;
    out->wait_d = hc.wait_cycles * inv;
    out->abort_d = hc.abort_cycles * inv;
    out->mng_d = hc.mng_cycles * inv;
    out->tot_d = hc.tot_cycles * inv;
    out->idx_d = hc.idx_cycles * inv;
    out->rank_count = gputx ? hc.max_rank + 1 : 0;
    out->batches = nlaunch;
    out->kernel_launches = e->kernel_launches - launches0;
    out->max_attempts = hc.max_attempts;
    out->err_site = hc.err_where;
    // latency percentiles from the histogram (bucket upper edges)
    out->lat_p50_us = hist_percentile_us(hc, 0.50);
    out->lat_p99_us = hist_percentile_us(hc, 0.99);
    if (hc.err) return (int)hc.err;
    if (hc.committed != e->n_tx) return GCC_ESTATE;
    return GCC_OK;
}

int gcc_load_var_txs(gcc_engine *e, const uint32_t *tx_off, const gcc_ycsb_req *reqs,
                     uint64_t n_tx) {
    cudaGetLastError();  // a stale error of an earlier call is not ours
    if (!e || !tx_off || (!reqs && n_tx)) return GCC_EINVAL;
    if (n_tx == 0 || n_tx >= (1ull << 27)) return GCC_EINVAL;
    if (tx_off[0] != 0) return GCC_EINVAL;
    for (uint64_t t = 0; t < n_tx; ++t)
        if (tx_off[t + 1] < tx_off[t] || tx_off[t + 1] - tx_off[t] > (uint32_t)kMaxVarOps)
            return GCC_EFORMAT;
    const uint64_t ops = tx_off[n_tx];
    cudaSetDevice(e->dev);
    int rc;
    if (e->cap_var < n_tx) {
        if ((rc = e->alloc(&e->tx_off_d, (n_tx + 1) * 4))) return rc;
        e->cap_var = n_tx;
    }
    if (e->cap_var_ops < ops) {
        if ((rc = e->alloc(&e->reqs_d, ops * sizeof(gcc_ycsb_req)))) return rc;
        e->cap_var_ops = ops;
    }
    if (e->cap_tx < n_tx) {
        if ((rc = e->alloc(&e->digest, n_tx * 8))) return rc;
        if ((rc = e->alloc(&e->commit_hi, n_tx * 8))) return rc;
        if ((rc = e->alloc(&e->commit_lo, n_tx * 8))) return rc;
        if ((rc = e->alloc(&e->tx_aborts, n_tx * 4))) return rc;
        e->cap_tx = n_tx;
    }
    if (!e->queue_tail && (rc = e->alloc(&e->queue_tail, 8))) return rc;
    cudaError_t ce = cudaMemcpyAsync(e->tx_off_d, tx_off, (n_tx + 1) * 4, cudaMemcpyHostToDevice, e->stream);
    if (ce == cudaSuccess && ops)
        ce = cudaMemcpyAsync(e->reqs_d, reqs, ops * sizeof(gcc_ycsb_req), cudaMemcpyHostToDevice, e->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
    if (ce != cudaSuccess) return e->fail_cuda(ce);
    e->tx_off_h.assign(tx_off, tx_off + n_tx + 1);
    e->n_var = n_tx;
    e->var_ops = ops;
    e->have_run = false;
    if (e->graph) {
        cudaGraphExecDestroy(e->graph);
        e->graph = nullptr;
        e->graph_key.clear();
    }
    return GCC_OK;
}

namespace {

// Schemes with variable-length kernels: every scheme but the ordered ones
// (GaccO / GPUTx build their per-row access orders from 16-slot records).
bool var_scheme(int s) {
    return s != S_GACCO && s != S_GPUTX && s >= 0 && s < S_COUNT;
}

// Autotuner candidates (warp_density, block_size, grid divisor, batch_size
// = transactions per launch inside a batch, 0 for the whole batch), tried in
// this order: the densest groups first, the same cut into launches of
// 65,536 / 16,384 (a barrier between launches drains the retry chains of hot
// rows, as the reference's batch loop does), then fewer transactions in
// flight, then more.
const int kArms[][4] = {{5, 32, 1, 0}, {5, 32, 2, 0}, {5, 32, 1, 65536}, {5, 32, 2, 16384},
                        {5, 32, 4, 0}, {4, 32, 2, 0}, {5, 16, 1, 0}, {4, 32, 1, 0},
                        {3, 32, 2, 0}, {3, 32, 1, 0}};

// Batch class: log2 of the batch size and the mean requests per tx in
// steps of 8.
int batch_class(const std::vector<uint32_t> &off, uint64_t t0, uint64_t t1) {
    uint64_t n = t1 - t0;
    int lg = 0;
    while ((1ull << (lg + 1)) <= n) ++lg;
    uint64_t ops = off[t1] - off[t0];
    int ob = (int)(n ? (ops / n) / 8 : 0);
    return lg * 16 + ob;
}

// Next config of a class: untried arms in order, then the fastest measured.
// An untried arm is skipped when a measured arm with no more transactions in
// flight already ran over 2x slower than the best: under contention adding
// transactions in flight only adds aborts, and one bad arm can cost 10-50x.
gcc_engine::Arm *pick_arm(std::vector<gcc_engine::Arm> &arms) {
    gcc_engine::Arm *best = nullptr;
    for (auto &a : arms)
        if (a.runs && (!best || a.ms_per_tx < best->ms_per_tx)) best = &a;
    for (auto &a : arms) {
        if (a.runs) continue;
        bool pruned = false;
        for (auto &m : arms)
            if (best && m.runs && m.active <= a.active && m.ms_per_tx > 2.0 * best->ms_per_tx)
                pruned = true;
        if (!pruned) return &a;
    }
    return best ? best : &arms[0];
}

__global__ void k_set_u64(unsigned long long *p, unsigned long long v) { *p = v; }

}  // namespace

int gcc_run_batches(gcc_engine *e, const gcc_run_params *rp, const uint32_t *batch_off,
                    uint64_t nb, int32_t mode, gcc_result *out) {
    cudaGetLastError();  // a stale error of an earlier call is not ours
    if (!e || !rp || !batch_off || !out || nb == 0) return GCC_EINVAL;
    memset(out, 0, sizeof(*out));
    const int s = gcc_scheme_id(rp->cc_scheme);
    if (s < 0 || !var_scheme(s)) return GCC_EINVAL;
    if (mode != GCC_BATCHES_SEQUENTIAL && mode != GCC_BATCHES_QUEUE) return GCC_EINVAL;
    if (mode == GCC_BATCHES_QUEUE && is_mvcc(s)) return GCC_EINVAL;
    if (rp->warp_density < 2 || rp->warp_density > 5) return GCC_EINVAL;
    if (rp->block_size < 1 || rp->block_size > 32) return GCC_EINVAL;
    if (rp->write_mode != GCC_WRITE_FIELD) return GCC_EINVAL;
    if (!ext_ops_allowed(e, s, rp)) return GCC_EINVAL;
    if (rp->backoff_ns < -1 || rp->backoff_ns > 100000) return GCC_EINVAL;
    if (!e->n_var || !e->reqs_d) return GCC_ESTATE;
    if (batch_off[0] != 0 || batch_off[nb] != e->n_var) return GCC_EINVAL;
    for (uint64_t b = 0; b < nb; ++b)
        if (batch_off[b + 1] <= batch_off[b]) return GCC_EINVAL;
    cudaSetDevice(e->dev);
    const bool autotune = (rp->flags & GCC_F_AUTOTUNE) != 0;
    const bool use_graph = (rp->flags & GCC_F_GRAPH) != 0;
    int rc;

    // per-batch (or whole-run) configuration
    const uint64_t nconf = mode == GCC_BATCHES_QUEUE ? 1 : nb;
    if (rp->max_active < 0 || rp->starve_limit < -1) return GCC_EINVAL;
    std::vector<int> wd(nconf, rp->warp_density), bs(nconf, rp->block_size), cls(nconf, -1);
    std::vector<int> dv(nconf, 1);
    std::vector<uint32_t> split(nconf, 0);
    if (autotune) {
        for (uint64_t b = 0; b < nconf; ++b) {
            cls[b] = mode == GCC_BATCHES_QUEUE ? -1 : batch_class(e->tx_off_h, batch_off[b], batch_off[b + 1]);
            auto &arms = e->tuner[cls[b]];
            if (arms.empty())
                for (auto &a : kArms) {
                    const int G = 1 << a[0], block = a[1] * 32;
                    const uint64_t full =
                        (uint64_t)std::max(0, occupancy_var(s, G, block)) * e->sm_count;
                    const uint64_t act = std::max<uint64_t>(1, full / a[2]) * (uint64_t)(block / G);
                    if (mode == GCC_BATCHES_QUEUE && a[3]) continue;  // one launch in queue mode
                    arms.push_back({a[0], a[1], a[2], (uint32_t)a[3], act, 0.0, 0});
                }
        }
        // one untried arm per class per run, so the runs of a class measure
        // the arms one by one and the class settles on its fastest
        std::map<int, gcc_engine::Arm *> chosen;
        for (uint64_t b = 0; b < nconf; ++b) {
            auto it = chosen.find(cls[b]);
            if (it == chosen.end()) it = chosen.emplace(cls[b], pick_arm(e->tuner[cls[b]])).first;
            wd[b] = it->second->wd;
            bs[b] = it->second->bs;
            dv[b] = it->second->div;
            split[b] = it->second->split;
        }
    }
    uint64_t max_batch = 0;
    for (uint64_t b = 0; b < nb; ++b) max_batch = std::max<uint64_t>(max_batch, batch_off[b + 1] - batch_off[b]);
    if (is_slow(s) && !e->latch) {
        if ((rc = e->alloc(&e->latch, e->rows * 4))) return rc;
        cudaError_t le = cudaMemsetAsync(e->latch, 0, e->rows * 4, e->stream);
        if (le != cudaSuccess) return e->fail_cuda(le);
    }
    if (is_mvcc(s) && e->ver_units * kMaxOps < max_batch * kMaxVarOps) {
        uint64_t nodes = max_batch * kMaxVarOps;
        if ((rc = e->alloc(&e->ver_ts, nodes * 8))) return rc;
        if ((rc = e->alloc(&e->ver_prev, nodes * 4))) return rc;
        if ((rc = e->alloc(&e->ver_data, nodes * e->wslot * 8))) return rc;
        e->ver_units = (nodes + kMaxOps - 1) / kMaxOps;
    }
    std::vector<int> grid(nconf), block(nconf);
    for (uint64_t b = 0; b < nconf; ++b) {
        block[b] = bs[b] * 32;
        const int G = 1 << wd[b];
        int occ = occupancy_var(s, G, block[b]);
        if (occ <= 0) return GCC_EINVAL;
        uint64_t n = mode == GCC_BATCHES_QUEUE ? e->n_var : batch_off[b + 1] - batch_off[b];
        uint64_t want = (n * (uint64_t)G + block[b] - 1) / block[b];
        uint64_t cap = std::max<uint64_t>(1, (uint64_t)occ * e->sm_count / dv[b]);
        if (!autotune) cap = std::min<uint64_t>(cap, active_grid(rp->max_active, G, block[b]));
        grid[b] = (int)std::max<uint64_t>(1, std::min<uint64_t>(want, cap));
    }
    const uint64_t nst = 3 * nb + 4;
    if (e->stamps_cap < nst) {
        if ((rc = e->alloc(&e->stamps, nst * 8))) return rc;
        e->stamps_cap = nst;
    }

    KParams p = e->base_params();
    p.txs = nullptr;
    p.tx_off = e->tx_off_d;
    p.reqs = e->reqs_d;
    p.n_tx = (uint32_t)e->n_var;
    p.slot_ops = kMaxVarOps;
    p.write_mode = rp->write_mode;
    p.write_seed = rp->write_seed;
    p.flags = rp->flags;
    p.spin_limit_ns = rp->spin_limit_ns ? rp->spin_limit_ns : 4000000000ull;
    p.backoff_ns = rp->backoff_ns < 0 ? 0u : (rp->backoff_ns == 0 ? 512u : (uint32_t)rp->backoff_ns);
    p.starve_limit = starve_param(rp->starve_limit);
    p.ordered_from = rp->ordered_after > 0 ? (uint32_t)rp->ordered_after + 1u : 0u;
    p.ext_ops = (rp->flags & GCC_F_EXT_OPS) ? 1u : 0u;
    p.ver_ts = e->ver_ts;
    p.ver_prev = e->ver_prev;
    p.ver_data = e->ver_data;

    // graph key: everything the captured work depends on
    std::vector<uint64_t> key = {(uint64_t)s, (uint64_t)mode, rp->flags, rp->write_seed,
                                 p.spin_limit_ns, p.backoff_ns, p.starve_limit, (uint64_t)e->n_var, nb};
    for (uint64_t b = 0; b <= nb; ++b) key.push_back(batch_off[b]);
    for (uint64_t b = 0; b < nconf; ++b) {
        key.push_back(((uint64_t)wd[b] << 48) | ((uint64_t)bs[b] << 32) | (uint64_t)grid[b]);
        key.push_back(split[b]);
    }
    // transaction-kernel launches of the run
    uint64_t launches = 0;
    if (mode == GCC_BATCHES_QUEUE) {
        launches = 1;
    } else {
        for (uint64_t b = 0; b < nb; ++b) {
            const uint64_t n = batch_off[b + 1] - batch_off[b];
            const uint64_t step = split[b] ? std::min<uint64_t>(split[b], n) : n;
            launches += (n + step - 1) / step;
        }
    }

    cudaStream_t st = e->stream;
    unsigned long long *stamp = e->stamps;
    auto mark = [&](int i) -> cudaError_t {
        k_stamp<<<1, 1, 0, st>>>(stamp, i);
        return cudaGetLastError();
    };
    const bool needs_reset = uses_ts(s) || !(rp->flags & GCC_F_NO_RESET);
    auto enqueue = [&]() -> cudaError_t {
        cudaError_t ce = cudaMemsetAsync(e->ctr, 0, sizeof(Counters), st);
        if (ce == cudaSuccess) ce = mark(0);
        if (mode == GCC_BATCHES_QUEUE) {
            // one reset, every batch admitted to the queue, one persistent
            // launch that drains positions 0..n_var-1 in order
            if (ce == cudaSuccess) ce = cudaMemsetAsync(e->meta, 0, e->rows * 8, st);
            if (ce == cudaSuccess) {
                k_batch_prep<<<1, 32, 0, st>>>(e->ctr, uses_ts(s) ? 1 : 0);
                k_set_u64<<<1, 1, 0, st>>>(e->queue_tail, e->n_var);
                ce = cudaGetLastError();
            }
            KParams q = p;
            q.batch_st = 0;
            q.batch_n = (uint32_t)e->n_var;
            q.queue_tail = e->queue_tail;
            if (ce == cudaSuccess) ce = mark(3);
            if (ce == cudaSuccess) ce = launch_var(s, 1 << wd[0], grid[0], block[0], q, st);
            if (ce == cudaSuccess) ce = mark(4);
        } else {
            for (uint64_t b = 0; b < nb && ce == cudaSuccess; ++b) {
                KParams q = p;
                q.batch_st = batch_off[b];
                q.batch_n = batch_off[b + 1] - batch_off[b];
                ce = mark(3 + 3 * (int)b);
                if (ce == cudaSuccess && (needs_reset || b == 0))
                    ce = cudaMemsetAsync(e->meta, 0, e->rows * 8, st);
                if (ce == cudaSuccess && is_mvcc(s)) ce = cudaMemsetAsync(e->turn, 0xFF, e->rows * 4, st);
                if (ce == cudaSuccess) {
                    k_batch_prep<<<1, 32, 0, st>>>(e->ctr, uses_ts(s) ? 1 : 0);
                    ce = cudaGetLastError();
                }
                if (ce == cudaSuccess) ce = mark(4 + 3 * (int)b);
                // the batch in launches of at most split[b] transactions
                // (the tickets restart per launch; timestamps and metadata
                // carry on inside the batch)
                const uint32_t bn = q.batch_n;
                const uint32_t step = split[b] ? std::min<uint32_t>(split[b], bn) : bn;
                for (uint32_t o = 0; o < bn && ce == cudaSuccess; o += step) {
                    KParams r = q;
                    r.batch_st = q.batch_st + o;
                    r.batch_n = std::min<uint32_t>(step, bn - o);
                    if (o) {
                        k_batch_prep<<<1, 32, 0, st>>>(e->ctr, 0);
                        ce = cudaGetLastError();
                    }
                    if (ce == cudaSuccess) ce = launch_var(s, 1 << wd[b], grid[b], block[b], r, st);
                }
                if (ce == cudaSuccess) ce = mark(5 + 3 * (int)b);
            }
        }
        if (ce == cudaSuccess) ce = mark(2);
        return ce;
    };
    cudaError_t ce = cudaSuccess;
    if (use_graph) {
        if (!e->graph || e->graph_key != key) {
            if (e->graph) {
                cudaGraphExecDestroy(e->graph);
                e->graph = nullptr;
            }
            cudaGraph_t gr = nullptr;
            ce = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
            if (ce == cudaSuccess) {
                cudaError_t ce2 = enqueue();
                ce = cudaStreamEndCapture(st, &gr);
                if (ce2 != cudaSuccess) ce = ce2;
            }
            if (ce == cudaSuccess) ce = cudaGraphInstantiate(&e->graph, gr, 0);
            if (gr) cudaGraphDestroy(gr);
            if (ce != cudaSuccess) {
                e->graph = nullptr;
                return e->fail_cuda(ce);
            }
            e->graph_key = key;
        }
        ce = cudaGraphLaunch(e->graph, st);
    } else {
        ce = enqueue();
    }
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
    if (ce != cudaSuccess) return e->fail_cuda(ce);

    Counters hc;
    ce = cudaMemcpy(&hc, e->ctr, sizeof(Counters), cudaMemcpyDeviceToHost);
    if (ce != cudaSuccess) return e->fail_cuda(ce);
    std::vector<unsigned long long> ts(nst, 0);
    ce = cudaMemcpy(ts.data(), e->stamps, nst * 8, cudaMemcpyDeviceToHost);
    if (ce != cudaSuccess) return e->fail_cuda(ce);
    auto span_ms = [&](int a, int b) { return ts[b] > ts[a] ? (double)(ts[b] - ts[a]) * 1e-6 : 0.0; };
    e->have_run = true;
    e->n_tx = e->n_var;  // outputs are indexed by the variable-length txs now
    double proc = 0, pre = 0;
    e->bstat_wd.assign(nconf, 0);
    e->bstat_bs.assign(nconf, 0);
    e->bstat_ms.assign(nconf, 0.0);
    e->bstat_active.assign(nconf, 0);
    e->bstat_split.assign(nconf, 0);
    for (uint64_t b = 0; b < nconf; ++b) {
        double kms;
        if (mode == GCC_BATCHES_QUEUE) {
            kms = span_ms(3, 4);
        } else {
            pre += span_ms(3 + 3 * (int)b, 4 + 3 * (int)b);
            kms = span_ms(4 + 3 * (int)b, 5 + 3 * (int)b);
        }
        proc += kms;
        e->bstat_wd[b] = wd[b];
        e->bstat_bs[b] = bs[b];
        e->bstat_ms[b] = kms;
        e->bstat_active[b] = (uint64_t)grid[b] * (uint64_t)(block[b] >> wd[b]);
        e->bstat_split[b] = split[b];
    }
    const double tot_ms = span_ms(0, 2);
    if (autotune && !hc.err) {
        // feed the tuner: kernel ms per transaction of each class's arm
        std::map<int, std::pair<double, uint64_t>> agg;
        for (uint64_t b = 0; b < nconf; ++b) {
            uint64_t n = mode == GCC_BATCHES_QUEUE ? e->n_var : batch_off[b + 1] - batch_off[b];
            auto &a = agg[cls[b]];
            a.first += e->bstat_ms[b];
            a.second += n;
        }
        for (auto &kv : agg) {
            auto &arms = e->tuner[kv.first];
            for (auto &a : arms) {
                if (a.wd != wd[0] && mode == GCC_BATCHES_QUEUE) continue;
                bool match = false;
                for (uint64_t b = 0; b < nconf; ++b)
                    if (cls[b] == kv.first && wd[b] == a.wd && bs[b] == a.bs && dv[b] == a.div &&
                        split[b] == a.split)
                        match = true;
                if (!match) continue;
                double v = kv.second.first / (double)kv.second.second;
                a.ms_per_tx = a.runs ? 0.5 * (a.ms_per_tx + v) : v;
                a.runs += 1;
            }
        }
    }
    e->last_kernel_ms = proc;
    e->last_launches = nconf;
    out->committed = hc.committed;
    out->aborts = hc.aborts;
    out->pre_s = pre / 1000.0;
    out->proc_s = proc / 1000.0;
    out->tot_s = tot_ms / 1000.0;
    out->tx_per_s = tot_ms > 0 ? (double)hc.committed * 1000.0 / tot_ms : 0.0;
    const double inv = 1.0 / ((double)e->n_var * (double)e->clock_khz);
    out->ts_d = hc.ts_cycles * inv;
    out->wait_d = hc.wait_cycles * inv;
    out->abort_d = hc.abort_cycles * inv;
    out->mng_d = hc.mng_cycles * inv;
    out->tot_d = hc.tot_cycles * inv;
    out->idx_d = hc.idx_cycles * inv;
    out->batches = nb;
    // transaction kernels + per-batch prep (+ the queue tail write)
    out->kernel_launches = mode == GCC_BATCHES_QUEUE ? launches + 2 : 2 * launches;
    out->max_attempts = hc.max_attempts;
    out->err_site = hc.err_where;
    out->lat_p50_us = hist_percentile_us(hc, 0.50);
    out->lat_p99_us = hist_percentile_us(hc, 0.99);
    if (hc.err) return (int)hc.err;
    if (hc.committed != e->n_var) return GCC_ESTATE;
    return GCC_OK;
}

int gcc_get_batch_split(gcc_engine *e, uint32_t *split, uint64_t n) {
    if (!e || !split || n > e->bstat_split.size()) return GCC_EINVAL;
    std::copy(e->bstat_split.begin(), e->bstat_split.begin() + n, split);
    return GCC_OK;
}

int gcc_get_batch_active(gcc_engine *e, uint64_t *active, uint64_t n) {
    if (!e || !active) return GCC_EINVAL;
    if (!e->have_run || n > e->bstat_active.size()) return GCC_ESTATE;
    for (uint64_t i = 0; i < n; ++i) active[i] = e->bstat_active[i];
    return GCC_OK;
}

int gcc_get_batch_stats(gcc_engine *e, int32_t *wd, int32_t *bs, double *kms, uint64_t n) {
    if (!e || !wd || !bs || !kms) return GCC_EINVAL;
    if (!e->have_run || n > e->bstat_ms.size()) return GCC_ESTATE;
    for (uint64_t i = 0; i < n; ++i) {
        wd[i] = e->bstat_wd[i];
        bs[i] = e->bstat_bs[i];
        kms[i] = e->bstat_ms[i];
    }
    return GCC_OK;
}

int gcc_run_host(gcc_engine *e, const gcc_run_params *rp, const gcc_ycsb_tx *host_txs,
                 uint64_t n_tx, uint64_t *host_digests, gcc_result *out) {
    cudaGetLastError();
    if (!e || !rp || !host_txs || !out || n_tx == 0) return GCC_EINVAL;
    if (n_tx >= (1ull << 27)) return GCC_EINVAL;
    cudaSetDevice(e->dev);
    int rc = reserve_records(e, n_tx);
    if (rc) return rc;
    e->n_tx = n_tx;
    e->n_rec = n_tx;
    e->have_run = false;
    e->host_src = host_txs;
    e->host_dg = host_digests;
    rc = gcc_run(e, rp, out);
    e->host_src = nullptr;
    e->host_dg = nullptr;
    return rc;
}

int gcc_run_checked(gcc_engine *e, const gcc_run_params *rp, gcc_result *out, int *verdict) {
    cudaGetLastError();  // a stale error of an earlier call is not ours
    if (!e || !rp || !out || !verdict) return GCC_EINVAL;
    *verdict = 0;
    if (!e->txs || e->n_rec == 0) return GCC_ESTATE;
    e->n_tx = e->n_rec;
    cudaSetDevice(e->dev);
    const size_t tbytes = e->rows * e->stride;
    const uint64_t n = e->n_tx;
    uint8_t *snap = nullptr, *final_t = nullptr;
    unsigned long long *final_dg = nullptr, *diff = nullptr;
    uint32_t *order_d = nullptr;
    int rc = GCC_OK;
    cudaError_t ce = cudaMalloc(&snap, tbytes);
    if (ce == cudaSuccess) ce = cudaMalloc(&final_t, tbytes);
    if (ce == cudaSuccess) ce = cudaMalloc(&final_dg, n * 8);
    if (ce == cudaSuccess) ce = cudaMalloc(&diff, 8);
    if (ce == cudaSuccess) ce = cudaMalloc(&order_d, n * 4);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(snap, e->table, tbytes, cudaMemcpyDeviceToDevice, e->stream);
    gcc_run_params p = *rp;
    p.flags |= GCC_F_COMMIT_LOG;
    if (ce == cudaSuccess) {
        rc = gcc_run(e, &p, out);
        if (rc == GCC_OK) {
            std::vector<gcc_commit_rec> log(n);
            rc = gcc_get_commit_log(e, log.data(), n);
            std::vector<uint32_t> order(n);
            for (uint64_t i = 0; i < n; ++i) order[i] = (uint32_t)i;
            std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
                if (log[a].hi != log[b].hi) return log[a].hi < log[b].hi;
                if (log[a].lo != log[b].lo) return log[a].lo < log[b].lo;
                return a < b;
            });
            cudaStream_t st = e->stream;
            ce = cudaMemcpyAsync(final_t, e->table, tbytes, cudaMemcpyDeviceToDevice, st);
            if (ce == cudaSuccess) ce = cudaMemcpyAsync(final_dg, e->digest, n * 8, cudaMemcpyDeviceToDevice, st);
            if (ce == cudaSuccess) ce = cudaMemcpyAsync(order_d, order.data(), n * 4, cudaMemcpyHostToDevice, st);
            if (ce == cudaSuccess) ce = cudaMemcpyAsync(e->table, snap, tbytes, cudaMemcpyDeviceToDevice, st);
            if (ce == cudaSuccess) ce = cudaMemsetAsync(e->ctr, 0, sizeof(Counters), st);
            // replay: one ordered launch over every transaction in log order
            KParams q = e->base_params();
            q.write_mode = rp->write_mode;
            q.write_seed = rp->write_seed;
            q.spin_limit_ns = rp->spin_limit_ns ? rp->spin_limit_ns : 4000000000ull;
            q.order = order_d;
            q.batch_st = 0;
            q.batch_n = (uint32_t)n;
            if (rp->write_mode == GCC_WRITE_ROWCOPY && e->scratch_units < n) {
                rc = e->alloc(&e->scratch, n * kMaxOps * e->wslot * 8);
                e->scratch_units = rc ? 0 : n;
            }
            q.scratch = rp->write_mode == GCC_WRITE_ROWCOPY ? e->scratch : nullptr;
            if (ce == cudaSuccess && rc == GCC_OK) rc = e->order_pass(q, n, 0);
            q.op_row = e->op_row;
            q.op_pos = e->op_pos;
            if (ce == cudaSuccess && rc == GCC_OK) {
                const int block = 256;
                int occ = scheme_occupancy(S_GACCO, 32, block);
                int grid = (int)std::max<uint64_t>(1, std::min<uint64_t>((n * 32 + block - 1) / block,
                                                                       (uint64_t)occ * e->sm_count));
                k_batch_prep<<<1, 32, 0, st>>>(e->ctr, 0);
                ce = launch_scheme_kernel(S_GACCO, 32, grid, block, q, st);
            }
            unsigned long long d_t = 0, d_d = 0;
            if (ce == cudaSuccess) ce = cudaMemsetAsync(diff, 0, 8, st);
            if (ce == cudaSuccess) {
                k_count_diff<<<1024, 256, 0, st>>>((const unsigned long long *)final_t,
                                                   (const unsigned long long *)e->table, tbytes / 8, diff);
                ce = cudaMemcpyAsync(&d_t, diff, 8, cudaMemcpyDeviceToHost, st);
            }
            if (ce == cudaSuccess) ce = cudaMemsetAsync(diff, 0, 8, st);
            if (ce == cudaSuccess) {
                k_count_diff<<<256, 256, 0, st>>>(final_dg, e->digest, n, diff);
                ce = cudaMemcpyAsync(&d_d, diff, 8, cudaMemcpyDeviceToHost, st);
            }
            unsigned err = 0;
            if (ce == cudaSuccess) ce = cudaMemcpyAsync(&err, &e->ctr->err, 4, cudaMemcpyDeviceToHost, st);
            if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
            if (ce == cudaSuccess && rc == GCC_OK) {
                if (err) rc = (int)err;
                *verdict = (!err && d_t == 0 && d_d == 0) ? 1 : 0;
            }
            // leave the engine in the checked run's final state
            if (ce == cudaSuccess) ce = cudaMemcpyAsync(e->table, final_t, tbytes, cudaMemcpyDeviceToDevice, st);
            if (ce == cudaSuccess) ce = cudaMemcpyAsync(e->digest, final_dg, n * 8, cudaMemcpyDeviceToDevice, st);
            if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
        }
    }
    cudaFree(snap);
    cudaFree(final_t);
    cudaFree(final_dg);
    cudaFree(diff);
    cudaFree(order_d);
    if (ce != cudaSuccess) return e->fail_cuda(ce);
    return rc;
}

int gcc_format_line(const gcc_run_params *p, const gcc_result *r, char *buf, size_t n) {
    if (!p || !r || !buf || n == 0) return GCC_EINVAL;
    // ExecInfo::Analyse writes floats through std::ostream (6 significant
    // digits); the same stream formatting is used here.
    std::ostringstream of;
    of << p->cc_scheme << "," << p->warp_density << "," << p->block_size << "," << p->batch_size
       << "," << (float)r->tx_per_s << "," << r->aborts << "," << (float)r->ts_d << ","
       << (float)r->wait_d << "," << (float)r->abort_d << "," << (float)r->mng_d << ","
       << (float)r->tot_d << "," << (float)r->idx_d << "," << (float)r->pre_s << ","
       << (float)r->proc_s << "," << (float)r->tot_s;
    std::string str = of.str();
    if (str.size() + 1 > n) return GCC_EINVAL;
    memcpy(buf, str.c_str(), str.size() + 1);
    return GCC_OK;
}

int gcc_dump_table(gcc_engine *e, void *dst, uint64_t bytes) {
    if (!e || !dst || bytes < e->rows * e->row_bytes) return GCC_EINVAL;
    cudaSetDevice(e->dev);
    cudaError_t ce = cudaMemcpy2DAsync(dst, e->row_bytes, e->table, e->stride, e->row_bytes,
                                       e->rows, cudaMemcpyDeviceToHost, e->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
    return ce == cudaSuccess ? GCC_OK : e->fail_cuda(ce);
}

}  // extern "C"

namespace {

// Initial order-entry rows (see gcc_oe_fill): one thread per row.
__global__ void k_oe_fill(uint8_t *table, uint64_t rows, uint32_t stride, gcc_oe_layout L,
                          uint64_t seed) {
    const uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (r >= rows) return;
    unsigned long long f[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    auto h = [&](uint32_t k) { return hash3(seed, r, k); };
    if (r < L.district) {
        f[0] = 30000000ull; f[1] = h(1) % 2001ull;
    } else if (r < L.customer) {
        f[0] = 3000000ull; f[1] = h(1) % 2001ull; f[2] = 3001ull;
    } else if (r < L.item) {
        f[0] = (unsigned long long)(-1000ll); f[1] = 1000ull; f[2] = 1ull; f[3] = h(3) % 5001ull;
    } else if (r < L.stock) {
        f[0] = 100ull + h(0) % 9901ull;
    } else if (r < L.inserts) {
        f[0] = 10ull + h(0) % 91ull;
    }
    unsigned long long *w = (unsigned long long *)(table + r * stride);
    w[0] = r;
#pragma unroll
    for (int k = 0; k < 10; ++k) w[1 + k] = f[k];
    for (uint32_t k = 11; k < stride / 8; ++k) w[k] = 0ull;
}

}  // namespace

extern "C" {

int gcc_oe_fill(gcc_engine *e, const gcc_oe_desc *d, uint64_t seed) {
    cudaGetLastError();
    if (!e || !d) return GCC_EINVAL;
    if (e->desc.layout != GCC_LAYOUT_U64X11) return GCC_EINVAL;
    gcc_oe_layout L;
    std::vector<uint32_t> off(2);
    int rc = gcc_oe_offsets(d, 0, seed, off.data(), &L);
    if (rc) return rc;
    if (e->rows < L.rows) return GCC_EINVAL;
    cudaSetDevice(e->dev);
    k_oe_fill<<<(unsigned)((e->rows + 255) / 256), 256, 0, e->stream>>>(e->table, e->rows, e->stride,
                                                                      L, seed);
    e->kernel_launches += 1;
    cudaError_t ce = cudaGetLastError();
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
    return ce == cudaSuccess ? GCC_OK : e->fail_cuda(ce);
}

int gcc_upload_table(gcc_engine *e, const void *src, uint64_t bytes) {
    if (!e || !src || bytes < e->rows * e->row_bytes) return GCC_EINVAL;
    cudaSetDevice(e->dev);
    cudaError_t ce = cudaMemcpy2DAsync(e->table, e->stride, src, e->row_bytes, e->row_bytes,
                                       e->rows, cudaMemcpyHostToDevice, e->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
    return ce == cudaSuccess ? GCC_OK : e->fail_cuda(ce);
}

static int copy_out(gcc_engine *e, void *dst, const void *src, uint64_t bytes) {
    if (!e->have_run) return GCC_ESTATE;
    cudaSetDevice(e->dev);
    cudaError_t ce = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, e->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
    return ce == cudaSuccess ? GCC_OK : e->fail_cuda(ce);
}

int gcc_get_digests(gcc_engine *e, uint64_t *dst, uint64_t n) {
    if (!e || !dst || n > e->n_tx) return GCC_EINVAL;
    return copy_out(e, dst, e->digest, n * 8);
}

int gcc_get_tx_aborts(gcc_engine *e, uint32_t *dst, uint64_t n) {
    if (!e || !dst || n > e->n_tx) return GCC_EINVAL;
    return copy_out(e, dst, e->tx_aborts, n * 4);
}

int gcc_get_commit_log(gcc_engine *e, gcc_commit_rec *dst, uint64_t n) {
    if (!e || !dst || n > e->n_tx) return GCC_EINVAL;
    std::vector<uint64_t> hi(n), lo(n);
    int rc = copy_out(e, hi.data(), e->commit_hi, n * 8);
    if (rc) return rc;
    if ((rc = copy_out(e, lo.data(), e->commit_lo, n * 8))) return rc;
    for (uint64_t i = 0; i < n; ++i) dst[i] = gcc_commit_rec{hi[i], lo[i]};
    return GCC_OK;
}

int gcc_get_read_log(gcc_engine *e, void *dst, uint64_t bytes) {
    if (!e || !dst) return GCC_EINVAL;
    uint64_t need = e->n_tx * kMaxOps * e->wslot * 8;
    if (!e->read_log || e->read_log_units < e->n_tx) return GCC_ESTATE;
    if (bytes < need) return GCC_EINVAL;
    return copy_out(e, dst, e->read_log, need);
}

int gcc_index_lookup(gcc_engine *e, const uint32_t *keys, uint32_t *rows, uint64_t n) {
    if (!e || (!keys && n) || (!rows && n)) return GCC_EINVAL;
    if (n == 0) return GCC_OK;
    cudaSetDevice(e->dev);
    uint32_t *dk = nullptr, *dr = nullptr;
    cudaError_t ce = cudaMalloc(&dk, n * 4);
    if (ce == cudaSuccess) ce = cudaMalloc(&dr, n * 4);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(dk, keys, n * 4, cudaMemcpyHostToDevice, e->stream);
    if (ce == cudaSuccess) {
        KParams p = e->base_params();
        k_index_lookup<<<grid1d(n, 256), 256, 0, e->stream>>>(p, dk, dr, n);
        ce = cudaGetLastError();
    }
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(rows, dr, n * 4, cudaMemcpyDeviceToHost, e->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
    if (dk) cudaFree(dk);
    if (dr) cudaFree(dr);
    return ce == cudaSuccess ? GCC_OK : e->fail_cuda(ce);
}

int gcc_last_kernel_ms(gcc_engine *e, double *kernel_ms, uint64_t *launches) {
    if (!e || !kernel_ms || !launches) return GCC_EINVAL;
    if (!e->have_run) return GCC_ESTATE;
    *kernel_ms = e->last_kernel_ms;
    *launches = e->last_launches;
    return GCC_OK;
}

}  // extern "C"

// ===========================================================================
// Learned contention scheduling (gcc_sched_*): the per-batch driver around
// the predictor of sched.cu. Each batch: features -> forward -> stable
// partition by predicted risk (device) -> policy choice (host, per
// contention bucket) -> one launch (plain ordering) or two (predicted-safe
// transactions at full concurrency, then the deferred ones with a cap on
// transactions in flight) -> the batch's requests enter the frequency table.
// Every explore_every-th batch first runs a probe of probe_rows transactions
// with plain ordering at full concurrency: their abort outcomes are the
// training labels (Adam steps follow) and their abort rate the yardstick.
// ===========================================================================
namespace {

struct SchedArm {
    uint32_t cap;      // in-flight cap of the deferred sub-batch (0: none)
    uint32_t wd;       // 1: deferred sub-batch under 2PL wait-die
    uint32_t defer;    // 0: plain ordering, one launch
};

constexpr int kSchedBuckets = 4;

// Contention bucket of a batch from its mean predicted abort probability.
int contention_bucket(double pm) {
    return std::max(0, std::min(kSchedBuckets - 1, (int)(pm * kSchedBuckets)));
}

}  // namespace

struct gcc_sched {
    gcc_engine *e = nullptr;
    gcc_sched_params prm{};
    sched::Predictor pred;
    uint32_t *order = nullptr;
    uint64_t order_cap = 0;
    uint32_t *part_scratch = nullptr;
    uint64_t part_cap = 0;
    uint32_t *counts = nullptr;
    float *sums = nullptr;
    unsigned long long *plan = nullptr;  // 2PL lock plans, by tx id
    uint64_t plan_cap = 0;
    std::vector<gcc_sched_batch> batches;
    // Policy: the arms of the scheme (0 = plain ordering, then deferral with
    // in-flight caps 2048 / 1024 / 512 / 256 / 128, then for 2PL wait-die at
    // 1024 and 512), an incumbent arm, and the arms compared with it since the
    // last refresh. A refresh happens when the mean prediction of a batch
    // has moved by more than 0.1 since the previous refresh (the contention
    // changed) or after 16 batches.
    std::vector<SchedArm> arms;
    int policy_scheme = -1;
    int inc = 0;
    std::vector<uint8_t> tried;
    uint32_t since_refresh = 0;
    float ref_pred = -1.f;
    ~gcc_sched() {
        if (e) cudaSetDevice(e->dev);
        void *bufs[] = {order, part_scratch, counts, sums, plan};
        for (void *b : bufs)
            if (b) cudaFree(b);
    }
    int fail(cudaError_t ce) {
        cudaGetLastError();
        return e->fail_cuda(ce);
    }
    void set_arms(int s) {
        arms.clear();
        arms.push_back({0u, 0u, 0u});
        for (uint32_t c : {2048u, 1024u, 512u, 256u, 128u}) arms.push_back({c, 0u, 1u});
        if (s == S_TPL_NW || s == S_TPL_WD)
            for (uint32_t c : {1024u, 512u}) arms.push_back({c, 1u, 1u});
        inc = 0;
        tried.assign(arms.size(), 0);
        since_refresh = 0;
        ref_pred = -1.f;
        policy_scheme = s;
    }
    // Candidate to compare against the incumbent for a batch whose mean
    // prediction is pm, or -1: the next larger or smaller cap (plain ordering
    // counts as the largest), then the wait-die arm at the incumbent's cap.
    int candidate(float pm) {
        if (++since_refresh > 16 || std::fabs(pm - ref_pred) > 0.1f) {
            std::fill(tried.begin(), tried.end(), 0);
            since_refresh = 0;
            ref_pred = pm;
        }
        const SchedArm &a = arms[inc];
        auto plain_cap_arm = [&](uint32_t cap) -> int {
            for (int k = 0; k < (int)arms.size(); ++k)
                if (!arms[k].wd && (arms[k].defer ? arms[k].cap : 0u) == cap) return k;
            return -1;
        };
        static const uint32_t kCaps[] = {0u, 2048u, 1024u, 512u, 256u, 128u};
        constexpr int kNumCaps = 6;
        int r = 0;
        const uint32_t mycap = a.defer ? a.cap : 0u;
        while (r < kNumCaps && kCaps[r] != mycap) ++r;
        for (int nr : {r + 1, r - 1}) {
            if (nr < 0 || nr >= kNumCaps) continue;
            const int k = plain_cap_arm(kCaps[nr]);
            if (k >= 0 && k != inc && !tried[k]) return k;
        }
        for (int k = 0; k < (int)arms.size(); ++k)
            if (arms[k].wd != a.wd && arms[k].cap == mycap && arms[k].defer && k != inc && !tried[k])
                return k;
        return -1;
    }
};

extern "C" {

uint64_t gcc_sched_param_count(void) { return (uint64_t)sched::kParams; }

int gcc_sched_create(gcc_engine *e, const gcc_sched_params *p, gcc_sched **out) {
    cudaGetLastError();
    if (!e || !p || !out) return GCC_EINVAL;
    *out = nullptr;
    if (p->mode != GCC_SCHED_PLAIN && p->mode != GCC_SCHED_LEARNED) return GCC_EINVAL;
    if (p->explore_every < 0 || p->minibatch < 0 || p->train_steps < -1 || p->probe_rows < 0 ||
        p->fixed_arm < 0 || p->min_sched < -1)
        return GCC_EINVAL;
    if (p->minibatch > (1 << 20) || p->probe_rows > (1 << 20)) return GCC_EINVAL;
    if (p->plan_threshold < -1 || p->plan_after < -1) return GCC_EINVAL;
    if (!(p->lr >= 0.f) || !(p->defer_threshold >= 0.f) || p->defer_threshold >= 1.f)
        return GCC_EINVAL;
    cudaSetDevice(e->dev);
    gcc_sched *s = new gcc_sched();
    s->e = e;
    s->prm = *p;
    if (!s->prm.explore_every) s->prm.explore_every = 4;
    if (!s->prm.train_steps) s->prm.train_steps = 4;
    if (!s->prm.minibatch) s->prm.minibatch = 4096;
    if (!s->prm.probe_rows) s->prm.probe_rows = 4096;
    if (!s->prm.min_sched) s->prm.min_sched = 4096;
    if (s->prm.lr == 0.f) s->prm.lr = 2e-3f;
    if (s->prm.defer_threshold == 0.f) s->prm.defer_threshold = 0.2f;
    if (!s->prm.plan_threshold) s->prm.plan_threshold = 1024;
    if (!s->prm.plan_after) s->prm.plan_after = 1;
    cudaError_t ce = s->pred.init(e->dev, e->stream,
                                  (uint64_t)std::max(4096, std::max(s->prm.minibatch, s->prm.probe_rows)),
                                  p->seed);
    if (ce == cudaSuccess) ce = cudaMalloc(&s->counts, 16);
    if (ce == cudaSuccess) ce = cudaMalloc(&s->sums, 16);
    if (ce != cudaSuccess) {
        int rc = s->fail(ce);
        delete s;
        return ce == cudaErrorMemoryAllocation ? GCC_ENOMEM : rc;
    }
    *out = s;
    return GCC_OK;
}

void gcc_sched_destroy(gcc_sched *s) { delete s; }

int gcc_sched_set_weights(gcc_sched *s, const float *w, uint64_t n) {
    if (!s || !w || n != (uint64_t)sched::kParams) return GCC_EINVAL;
    cudaSetDevice(s->e->dev);
    cudaError_t ce = s->pred.set_weights(w);
    return ce == cudaSuccess ? GCC_OK : s->fail(ce);
}

int gcc_sched_get_weights(gcc_sched *s, float *w, uint64_t n) {
    if (!s || !w || n != (uint64_t)sched::kParams) return GCC_EINVAL;
    cudaSetDevice(s->e->dev);
    cudaError_t ce = s->pred.get_weights(w);
    return ce == cudaSuccess ? GCC_OK : s->fail(ce);
}

int gcc_sched_features(gcc_sched *s, uint64_t first, uint64_t n, uint16_t *dst) {
    if (!s || (!dst && n) || n > (1ull << 20)) return GCC_EINVAL;
    gcc_engine *e = s->e;
    if (!e->txs || first + n > e->n_rec) return GCC_ESTATE;
    cudaSetDevice(e->dev);
    cudaError_t ce = s->pred.reserve(n);
    if (ce == cudaSuccess) ce = s->pred.features(e->txs, first, n, s->pred.feat);
    if (ce == cudaSuccess && n)
        ce = cudaMemcpyAsync(dst, s->pred.feat, n * sched::kFeatStride * 2, cudaMemcpyDeviceToHost,
                             e->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
    return ce == cudaSuccess ? GCC_OK : s->fail(ce);
}

int gcc_sched_lock_plans(gcc_sched *s, uint64_t first, uint64_t n, uint64_t *dst) {
    if (!s || (!dst && n) || n > (1ull << 20)) return GCC_EINVAL;
    gcc_engine *e = s->e;
    if (!e->txs || first + n > e->n_rec) return GCC_ESTATE;
    if (s->prm.plan_threshold <= 0) return GCC_EINVAL;
    cudaSetDevice(e->dev);
    cudaError_t ce = cudaSuccess;
    if (s->plan_cap < e->n_rec) {
        if (s->plan) cudaFree(s->plan);
        s->plan = nullptr;
        s->plan_cap = 0;
        ce = cudaMalloc(&s->plan, e->n_rec * 8);
        if (ce == cudaSuccess) s->plan_cap = e->n_rec;
    }
    if (ce == cudaSuccess)
        ce = s->pred.lock_plan(e->txs, first, n, (uint32_t)s->prm.plan_threshold, s->plan);
    if (ce == cudaSuccess && n)
        ce = cudaMemcpyAsync(dst, s->plan + first, n * 8, cudaMemcpyDeviceToHost, e->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
    return ce == cudaSuccess ? GCC_OK : s->fail(ce);
}

int gcc_sched_features_var(gcc_sched *s, uint64_t first, uint64_t n, uint16_t *dst) {
    if (!s || (!dst && n) || n > (1ull << 20)) return GCC_EINVAL;
    gcc_engine *e = s->e;
    if (!e->reqs_d || first + n > e->n_var) return GCC_ESTATE;
    cudaSetDevice(e->dev);
    cudaError_t ce = s->pred.reserve(n);
    if (ce == cudaSuccess) ce = s->pred.features_var(e->tx_off_d, e->reqs_d, first, n, s->pred.feat);
    if (ce == cudaSuccess && n)
        ce = cudaMemcpyAsync(dst, s->pred.feat, n * sched::kFeatStride * 2, cudaMemcpyDeviceToHost,
                             e->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
    return ce == cudaSuccess ? GCC_OK : s->fail(ce);
}

int gcc_sched_observe_var(gcc_sched *s, uint64_t first, uint64_t n, int32_t clear) {
    if (!s) return GCC_EINVAL;
    gcc_engine *e = s->e;
    if (n && (!e->reqs_d || first + n > e->n_var)) return GCC_ESTATE;
    cudaSetDevice(e->dev);
    cudaError_t ce = clear ? s->pred.clear_freq() : cudaSuccess;
    if (ce == cudaSuccess) ce = s->pred.observe_var(e->tx_off_d, e->reqs_d, first, n);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
    return ce == cudaSuccess ? GCC_OK : s->fail(ce);
}

int gcc_sched_observe(gcc_sched *s, uint64_t first, uint64_t n, int32_t clear) {
    if (!s) return GCC_EINVAL;
    gcc_engine *e = s->e;
    if (n && (!e->txs || first + n > e->n_rec)) return GCC_ESTATE;
    cudaSetDevice(e->dev);
    cudaError_t ce = clear ? s->pred.clear_freq() : cudaSuccess;
    if (ce == cudaSuccess) ce = s->pred.observe(e->txs, first, n);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
    return ce == cudaSuccess ? GCC_OK : s->fail(ce);
}

int gcc_sched_predict(gcc_sched *s, const uint16_t *feat, uint64_t n, float *p) {
    if (!s || !feat || !p || n == 0 || n > (1ull << 20)) return GCC_EINVAL;
    gcc_engine *e = s->e;
    cudaSetDevice(e->dev);
    cudaError_t ce = s->pred.reserve(n);
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(s->pred.feat, feat, n * sched::kFeatStride * 2, cudaMemcpyHostToDevice,
                             e->stream);
    if (ce == cudaSuccess) ce = s->pred.forward(s->pred.feat, n, s->pred.p);
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(p, s->pred.p, n * 4, cudaMemcpyDeviceToHost, e->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
    return ce == cudaSuccess ? GCC_OK : s->fail(ce);
}

static int sched_upload_rows(gcc_sched *s, const uint16_t *feat, const uint8_t *labels,
                             uint64_t n) {
    gcc_engine *e = s->e;
    cudaError_t ce = s->pred.reserve(n);
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(s->pred.feat, feat, n * sched::kFeatStride * 2, cudaMemcpyHostToDevice,
                             e->stream);
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(s->pred.labels, labels, n, cudaMemcpyHostToDevice, e->stream);
    return ce == cudaSuccess ? GCC_OK : s->fail(ce);
}

int gcc_sched_gradient(gcc_sched *s, const uint16_t *feat, const uint8_t *labels, uint64_t n,
                       float *grad, double *loss) {
    if (!s || !feat || !labels || !grad || n == 0 || n > (1ull << 20)) return GCC_EINVAL;
    gcc_engine *e = s->e;
    cudaSetDevice(e->dev);
    int rc = sched_upload_rows(s, feat, labels, n);
    if (rc) return rc;
    float lsum = 0.f;
    cudaError_t ce = s->pred.gradient(s->pred.feat, s->pred.labels, n);
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(grad, s->pred.grad, sched::kParams * 4, cudaMemcpyDeviceToHost, e->stream);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(&lsum, s->pred.loss, 4, cudaMemcpyDeviceToHost, e->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
    if (ce != cudaSuccess) return s->fail(ce);
    if (loss) *loss = (double)lsum / (double)n;
    return GCC_OK;
}

int gcc_sched_train(gcc_sched *s, const uint16_t *feat, const uint8_t *labels, uint64_t n,
                    int32_t steps, double *loss) {
    if (!s || !feat || !labels || n == 0 || n > (1ull << 20) || steps < 1) return GCC_EINVAL;
    gcc_engine *e = s->e;
    cudaSetDevice(e->dev);
    int rc = sched_upload_rows(s, feat, labels, n);
    if (rc) return rc;
    const uint64_t mb = std::min<uint64_t>(n, (uint64_t)s->prm.minibatch);
    cudaError_t ce = cudaSuccess;
    float lsum = 0.f;
    uint64_t rows = mb;
    for (int32_t k = 0; k < steps && ce == cudaSuccess; ++k) {
        const uint64_t off = ((uint64_t)k * mb) % n;
        rows = std::min<uint64_t>(mb, n - off);
        ce = s->pred.gradient(s->pred.feat + off * sched::kFeatStride, s->pred.labels + off, rows);
        if (ce == cudaSuccess) ce = s->pred.adam(s->prm.lr);
    }
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(&lsum, s->pred.loss, 4, cudaMemcpyDeviceToHost, e->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
    if (ce != cudaSuccess) return s->fail(ce);
    if (loss) *loss = (double)lsum / (double)rows;
    return GCC_OK;
}

int gcc_sched_batches(gcc_sched *s, gcc_sched_batch *dst, uint64_t n) {
    if (!s || (!dst && n)) return GCC_EINVAL;
    if (n > s->batches.size()) return GCC_ESTATE;
    for (uint64_t i = 0; i < n; ++i) dst[i] = s->batches[i];
    return GCC_OK;
}

}  // extern "C"

namespace {

// Per-run state of the scheduled driver, shared by gcc_sched_run (fixed
// batches of 16-request records) and gcc_serve (admitted batches of
// variable-length transactions).
struct SchedRun {
    gcc_sched *sc = nullptr;
    gcc_engine *e = nullptr;
    const gcc_run_params *rp = nullptr;
    int s = 0, G = 0, block = 0, occ_main = 0, occ_wd = 0;
    bool var = false, learned = false, planned = false;
    uint64_t user_grid = 0, batch_index = 0;
    KParams base;
    cudaEvent_t ev0, ev1, evk0, evk1, evt0, evt1, evp1, evq;
    double tot_ms = 0, proc_ms = 0, pred_ms = 0, train_ms = 0, probe_ms = 0, sched_ms = 0;
    uint64_t probe_c = 0, probe_a = 0, sched_c = 0, sched_a = 0;
    unsigned long long prev[2] = {0, 0};
    uint64_t launches0 = 0;
    std::vector<uint8_t> ylab;
};

// Validate the run, size the buffers for batches of up to max_batch
// transactions, reset the counters.
int sched_setup(SchedRun &R, gcc_sched *sc, const gcc_run_params *rp, bool var, uint64_t max_batch) {
    gcc_engine *e = sc->e;
    R.sc = sc;
    R.e = e;
    R.rp = rp;
    R.var = var;
    const int s = gcc_scheme_id(rp->cc_scheme);
    if (s != S_TPL_NW && s != S_TPL_WD && s != S_SILO && s != S_TICTOC) return GCC_EINVAL;
    if (rp->warp_density < (var ? 2 : 0) || rp->warp_density > 5) return GCC_EINVAL;
    if (rp->block_size < 1 || rp->block_size > 32) return GCC_EINVAL;
    if (rp->write_mode != GCC_WRITE_FIELD) return GCC_EINVAL;
    if (rp->flags & (GCC_F_READ_LOG | GCC_F_AUTOTUNE | GCC_F_GRAPH)) return GCC_EINVAL;
    if (!var && (rp->flags & GCC_F_EXT_OPS)) return GCC_EINVAL;
    if (!ext_ops_allowed(e, s, rp)) return GCC_EINVAL;
    if (rp->backoff_ns < -1 || rp->backoff_ns > 100000) return GCC_EINVAL;
    if (rp->max_active < 0 || rp->starve_limit < -1 || rp->ordered_after < 0) return GCC_EINVAL;
    if (max_batch == 0 || max_batch > (1ull << 20)) return GCC_EINVAL;
    cudaSetDevice(e->dev);
    R.s = s;
    R.learned = sc->prm.mode == GCC_SCHED_LEARNED;
    R.G = 1 << rp->warp_density;
    R.block = rp->block_size * 32;
    const uint64_t n = var ? e->n_var : e->n_rec;
    cudaError_t ce;
    if ((ce = sc->pred.reserve(max_batch))) return sc->fail(ce);
    if (sc->order_cap < n) {
        if (sc->order) cudaFree(sc->order);
        sc->order = nullptr;
        if ((ce = cudaMalloc(&sc->order, n * 4))) return sc->fail(ce);
        sc->order_cap = n;
    }
    // lock plans: 2PL on 16-request records
    R.planned = !var && (s == S_TPL_NW || s == S_TPL_WD) && sc->prm.plan_threshold > 0;
    if (R.planned && sc->plan_cap < n) {
        if (sc->plan) cudaFree(sc->plan);
        sc->plan = nullptr;
        if ((ce = cudaMalloc(&sc->plan, n * 8))) return sc->fail(ce);
        sc->plan_cap = n;
    }
    const uint64_t pneed = (max_batch + 1023) / 1024 * 3;
    if (sc->part_cap < pneed) {
        if (sc->part_scratch) cudaFree(sc->part_scratch);
        sc->part_scratch = nullptr;
        if ((ce = cudaMalloc(&sc->part_scratch, pneed * 4))) return sc->fail(ce);
        sc->part_cap = pneed;
    }
    R.occ_main = var ? occupancy_var(s, R.G, R.block) : scheme_occupancy(s, R.G, R.block);
    R.occ_wd = var ? occupancy_var(S_TPL_WD, R.G, R.block) : scheme_occupancy(S_TPL_WD, R.G, R.block);
    if (R.occ_main <= 0 || R.occ_wd <= 0) return GCC_EINVAL;
    if (sc->policy_scheme != s) sc->set_arms(s);
    KParams &b = R.base;
    b = e->base_params();
    if (var) {
        b.txs = nullptr;
        b.tx_off = e->tx_off_d;
        b.reqs = e->reqs_d;
        b.n_tx = (uint32_t)e->n_var;
        b.slot_ops = kMaxVarOps;
        b.ext_ops = (rp->flags & GCC_F_EXT_OPS) ? 1u : 0u;
    }
    b.write_mode = rp->write_mode;
    b.write_seed = rp->write_seed;
    b.flags = rp->flags;
    b.spin_limit_ns = rp->spin_limit_ns ? rp->spin_limit_ns : 4000000000ull;
    b.backoff_ns = rp->backoff_ns < 0 ? 0u : (rp->backoff_ns == 0 ? 512u : (uint32_t)rp->backoff_ns);
    b.starve_limit = starve_param(rp->starve_limit);
    b.ordered_from = rp->ordered_after > 0 ? (uint32_t)rp->ordered_after + 1u : 0u;
    R.user_grid = std::min<uint64_t>((uint64_t)R.occ_main * e->sm_count,
                                     active_grid(rp->max_active, R.G, R.block));
    int rc;
    if ((rc = e->ensure_events(8))) return rc;
    R.ev0 = e->events[0]; R.ev1 = e->events[1]; R.evk0 = e->events[2]; R.evk1 = e->events[3];
    R.evt0 = e->events[4]; R.evt1 = e->events[5]; R.evp1 = e->events[6]; R.evq = e->events[7];
    if ((ce = cudaMemsetAsync(e->ctr, 0, sizeof(Counters), e->stream))) return sc->fail(ce);
    R.launches0 = e->kernel_launches;
    e->n_tx = n;
    return GCC_OK;
}

// One batch (transactions bst .. bst + bn - 1) under the schedule; fills rec.
int sched_batch(SchedRun &R, uint64_t bst, uint64_t bn, gcc_sched_batch &rec) {
    gcc_sched *sc = R.sc;
    gcc_engine *e = R.e;
    const gcc_run_params *rp = R.rp;
    const int s = R.s, G = R.G, block = R.block;
    cudaStream_t st = e->stream;
    cudaError_t ce;
    auto launch = [&](int sch, uint64_t b0, uint64_t cnt, const uint32_t *order,
                      uint64_t grid_cap, bool planned = false) -> cudaError_t {
        KParams q = R.base;
        q.batch_st = (uint32_t)b0;
        q.batch_n = (uint32_t)cnt;
        q.order = order;
        q.wait_die = sch == S_TPL_WD ? 1u : 0u;
        if (planned) {
            q.plan = sc->plan;
            q.ordered_from = sc->prm.plan_after < 0 ? 1u : (uint32_t)sc->prm.plan_after + 1u;
        }
        k_batch_prep<<<1, 32, 0, st>>>(e->ctr, 0);
        cudaError_t c = cudaGetLastError();
        if (c != cudaSuccess) return c;
        const uint64_t want = (cnt * (uint64_t)G + block - 1) / block;
        const int grid = (int)std::max<uint64_t>(1, std::min<uint64_t>(want, grid_cap));
        e->kernel_launches += 2;
        return R.var ? launch_var(sch, G, grid, block, q, st)
                     : launch_scheme_kernel(sch, G, grid, block, q, st);
    };
    auto counters = [&](unsigned long long *ca) -> cudaError_t {
        cudaError_t c = cudaMemcpyAsync(ca, &e->ctr->committed, 16, cudaMemcpyDeviceToHost, st);
        return c == cudaSuccess ? cudaStreamSynchronize(st) : c;
    };
    // one part of a batch under an arm: plain ordering (one launch), or the
    // predicted-safe transactions at full concurrency then the deferred ones
    // with the arm's in-flight cap
    bool pl = false;  // scheduled 2PL batches run with lock plans (set below)
    auto run_part = [&](const SchedArm &a, uint64_t st0, uint64_t cnt, uint32_t n_low) -> cudaError_t {
        if (!cnt) return cudaSuccess;
        if (!a.defer) return launch(s, st0, cnt, nullptr, R.user_grid, pl);
        cudaError_t c = cudaSuccess;
        if (n_low) c = launch(s, st0, n_low, sc->order, R.user_grid, pl);
        if (c == cudaSuccess && cnt > n_low) {
            const int sch2 = a.wd ? S_TPL_WD : s;
            const int occ2 = a.wd ? R.occ_wd : R.occ_main;
            const uint64_t cap_grid = std::min<uint64_t>((uint64_t)occ2 * e->sm_count,
                                                         active_grid((int32_t)a.cap, G, block));
            c = launch(sch2, st0 + n_low, cnt - n_low, sc->order, cap_grid, pl);
        }
        return c;
    };
    const bool learned = R.learned && (sc->prm.min_sched < 0 || bn >= (uint64_t)sc->prm.min_sched);
    const uint64_t b = R.batch_index++;
    const uint64_t probe = (learned && b % (uint64_t)sc->prm.explore_every == 0)
                               ? std::min<uint64_t>(bn, (uint64_t)sc->prm.probe_rows) : 0;
    const uint64_t rst = bst + probe, rn = bn - probe;
    rec = gcc_sched_batch{};
    rec.kind = learned ? 1u : 0u;
    rec.probe = (uint32_t)probe;
    if ((ce = cudaEventRecord(R.ev0, st))) return sc->fail(ce);
    if (b == 0 || !(rp->flags & GCC_F_NO_RESET))
        if ((ce = cudaMemsetAsync(e->meta, 0, e->rows * 8, st))) return sc->fail(ce);
    // the part after the probe runs under the incumbent arm; when there is a
    // candidate, its second half runs under the candidate instead, so both
    // arms meet the same workload
    int arm_i = 0, cand = -1;
    uint64_t seg_n[2] = {rn, 0};
    uint32_t n_low[2] = {(uint32_t)rn, 0};
    float bpred_ms = 0;
    if (learned) {
        ce = R.var ? sc->pred.features_var(e->tx_off_d, e->reqs_d, bst, bn, sc->pred.feat)
                   : sc->pred.features(e->txs, bst, bn, sc->pred.feat);
        if (ce == cudaSuccess) ce = sc->pred.forward(sc->pred.feat, bn, sc->pred.p);
        e->kernel_launches += 4;  // features, 2 GEMMs + head
        if (ce == cudaSuccess && R.planned) {
            ce = sc->pred.lock_plan(e->txs, bst, bn, (uint32_t)sc->prm.plan_threshold, sc->plan);
            e->kernel_launches += 1;
            pl = true;
        }
        float hsums[4] = {0.f, 0.f, 0.f, 0.f};
        if (ce == cudaSuccess) {
            ce = sched::partition(sc->pred.p, bst, bn, sc->prm.defer_threshold, sc->order + bst,
                                  sc->counts, sc->sums, sc->part_scratch, st);
            e->kernel_launches += 3;
        }
        if (ce == cudaSuccess) ce = cudaMemcpyAsync(hsums, sc->sums, 8, cudaMemcpyDeviceToHost, st);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
        if (ce != cudaSuccess) return sc->fail(ce);
        rec.pred_mean = hsums[0] / (float)bn;
        rec.bucket = (uint32_t)contention_bucket(rec.pred_mean);
        if (sc->prm.fixed_arm > 0) {
            arm_i = std::min<int>(sc->prm.fixed_arm - 1, (int)sc->arms.size() - 1);
        } else {
            arm_i = sc->inc;
            cand = rn >= 2048 ? sc->candidate(rec.pred_mean) : -1;
        }
        if (cand >= 0) {
            seg_n[0] = rn / 2;
            seg_n[1] = rn - seg_n[0];
        }
        // risk partition of each part (positions keep their part)
        uint64_t off = rst;
        for (int k = 0; k < 2 && ce == cudaSuccess; ++k) {
            if (!seg_n[k]) continue;
            ce = sched::partition(sc->pred.p + (off - bst), off, seg_n[k], sc->prm.defer_threshold,
                                  sc->order + off, sc->counts + k, sc->sums + 2 * k,
                                  sc->part_scratch, st);
            e->kernel_launches += 3;
            off += seg_n[k];
        }
        if (ce == cudaSuccess) ce = cudaMemcpyAsync(n_low, sc->counts, 8, cudaMemcpyDeviceToHost, st);
        if (ce == cudaSuccess) ce = cudaEventRecord(R.evp1, st);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
        if (ce != cudaSuccess) return sc->fail(ce);
        if (!seg_n[1]) n_low[1] = 0;
        cudaEventElapsedTime(&bpred_ms, R.ev0, R.evp1);
        R.pred_ms += bpred_ms;
    }
    const SchedArm arm = sc->arms[arm_i];
    rec.arm = (uint32_t)arm_i;
    rec.explored = cand >= 0 ? (uint32_t)cand + 1u : 0u;
    rec.in_flight_cap = arm.defer ? arm.cap : 0u;
    rec.wait_die = arm.defer ? arm.wd : 0u;
    rec.deferred = (arm.defer ? seg_n[0] - n_low[0] : 0u) +
                   (cand >= 0 && sc->arms[cand].defer ? seg_n[1] - n_low[1] : 0u);

    // the probe: plain ordering at full concurrency, labels for training
    unsigned long long c_probe[2] = {R.prev[0], R.prev[1]};
    if (probe) {
        if ((ce = launch(s, bst, probe, nullptr, R.user_grid))) return sc->fail(ce);
        if ((ce = cudaEventRecord(R.evq, st))) return sc->fail(ce);
        if ((ce = counters(c_probe))) return sc->fail(ce);
        float qms = 0;
        cudaEventElapsedTime(&qms, R.evp1, R.evq);
        R.probe_ms += qms;
        R.probe_c += c_probe[0] - R.prev[0];
        R.probe_a += c_probe[1] - R.prev[1];
    }
    if ((ce = cudaEventRecord(R.evk0, st))) return sc->fail(ce);
    ce = run_part(arm, rst, seg_n[0], n_low[0]);
    if (ce == cudaSuccess) ce = cudaEventRecord(R.evt1, st);  // end of the first part
    if (ce == cudaSuccess && cand >= 0) ce = run_part(sc->arms[cand], rst + seg_n[0], seg_n[1], n_low[1]);
    if (ce == cudaSuccess) ce = cudaEventRecord(R.evk1, st);
    if (ce != cudaSuccess) return sc->fail(ce);
    float part_ms[2] = {0.f, 0.f};
    if (cand >= 0) {
        if ((ce = cudaEventSynchronize(R.evk1))) return sc->fail(ce);
        cudaEventElapsedTime(&part_ms[0], R.evk0, R.evt1);
        cudaEventElapsedTime(&part_ms[1], R.evt1, R.evk1);
    }
    const bool train = probe && sc->prm.train_steps > 0;
    if (train) {
        // labels of the probe, the loss of the predictions made before
        // training on them, then Adam steps
        ce = cudaEventRecord(R.evt0, st);
        if (ce == cudaSuccess) ce = sched::abort_labels(e->tx_aborts, bst, probe, sc->pred.labels, st);
        e->kernel_launches += 1;
        R.ylab.resize(probe);
        if (ce == cudaSuccess)
            ce = cudaMemcpyAsync(R.ylab.data(), sc->pred.labels, probe, cudaMemcpyDeviceToHost, st);
        const uint64_t mb = std::min<uint64_t>(probe, (uint64_t)sc->prm.minibatch);
        for (int32_t k = 0; k < sc->prm.train_steps && ce == cudaSuccess; ++k) {
            const uint64_t off = ((uint64_t)k * mb) % probe;
            const uint64_t rows = std::min<uint64_t>(mb, probe - off);
            ce = sc->pred.gradient(sc->pred.feat + off * sched::kFeatStride, sc->pred.labels + off, rows);
            if (ce == cudaSuccess && k == 0) {
                float l0 = 0.f;
                ce = cudaMemcpyAsync(&l0, sc->pred.loss, 4, cudaMemcpyDeviceToHost, st);
                if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
                rec.loss = l0 / (float)rows;
            }
            if (ce == cudaSuccess) ce = sc->pred.adam(sc->prm.lr);
            e->kernel_launches += 13;
        }
        if (ce == cudaSuccess) ce = cudaEventRecord(R.evt1, st);
        if (ce != cudaSuccess) return sc->fail(ce);
    }
    if (learned) {
        ce = R.var ? sc->pred.observe_var(e->tx_off_d, e->reqs_d, bst, bn)
                   : sc->pred.observe(e->txs, bst, bn);
        if (ce != cudaSuccess) return sc->fail(ce);
        e->kernel_launches += 2;
    }
    if ((ce = cudaEventRecord(R.ev1, st))) return sc->fail(ce);
    unsigned long long ca[2];
    if ((ce = counters(ca))) return sc->fail(ce);
    float ms = 0, kms = 0;
    cudaEventElapsedTime(&ms, R.ev0, R.ev1);
    cudaEventElapsedTime(&kms, R.evk0, R.evk1);
    if (train) {
        float tms = 0;
        cudaEventElapsedTime(&tms, R.evt0, R.evt1);
        R.train_ms += tms;
        uint64_t pos = 0;
        for (uint8_t v : R.ylab) pos += v;
        rec.label_mean = (float)pos / (float)probe;
    }
    rec.ms = ms;
    rec.committed = ca[0] - R.prev[0];
    rec.aborts = ca[1] - R.prev[1];
    R.tot_ms += ms;
    R.proc_ms += kms;
    R.sched_ms += kms;
    R.sched_c += ca[0] - c_probe[0];
    R.sched_a += ca[1] - c_probe[1];
    R.prev[0] = ca[0];
    R.prev[1] = ca[1];
    // the comparison: the candidate replaces the incumbent when its half
    // ran at least 3% faster per transaction
    if (cand >= 0) {
        sc->tried[cand] = 1;
        const double t_inc = part_ms[0] / (double)seg_n[0];
        const double t_cand = part_ms[1] / (double)seg_n[1];
        if (t_cand < 0.97 * t_inc) {
            sc->tried[arm_i] = 1;
            sc->inc = cand;
        }
    }
    unsigned err = 0;
    if (cudaMemcpy(&err, &e->ctr->err, 4, cudaMemcpyDeviceToHost) == cudaSuccess && err) return (int)err;
    return GCC_OK;
}

// Totals of the run into out (gcc_result and the scheduler's fields).
int sched_finish(SchedRun &R, uint64_t n, uint64_t nb, gcc_sched_result *out) {
    gcc_sched *sc = R.sc;
    gcc_engine *e = R.e;
    Counters hc;
    cudaError_t ce = cudaMemcpy(&hc, e->ctr, sizeof(Counters), cudaMemcpyDeviceToHost);
    if (ce != cudaSuccess) return sc->fail(ce);
    e->have_run = true;
    e->last_kernel_ms = R.proc_ms;
    e->last_launches = nb;
    gcc_result *r = &out->run;
    r->committed = hc.committed;
    r->aborts = hc.aborts;
    r->pre_s = (R.pred_ms + R.train_ms) / 1000.0;
    r->proc_s = (R.proc_ms + R.probe_ms) / 1000.0;
    r->tot_s = R.tot_ms / 1000.0;
    r->tx_per_s = R.tot_ms > 0 ? (double)hc.committed * 1000.0 / R.tot_ms : 0.0;
    const double inv = 1.0 / ((double)std::max<uint64_t>(1, n) * (double)e->clock_khz);
    r->ts_d = hc.ts_cycles * inv;
    r->wait_d = hc.wait_cycles * inv;
    r->abort_d = hc.abort_cycles * inv;
    r->mng_d = hc.mng_cycles * inv;
    r->tot_d = hc.tot_cycles * inv;
    r->idx_d = hc.idx_cycles * inv;
    r->batches = nb;
    r->kernel_launches = e->kernel_launches - R.launches0;
    r->max_attempts = hc.max_attempts;
    r->err_site = hc.err_where;
    r->lat_p50_us = hist_percentile_us(hc, 0.50);
    r->lat_p99_us = hist_percentile_us(hc, 0.99);
    for (auto &rec : sc->batches) {
        out->probed += rec.probe;
        out->deferred += rec.deferred;
        if (rec.probe && sc->prm.train_steps > 0) out->last_loss = rec.loss;
    }
    out->probe_tx_per_s = R.probe_ms > 0 ? R.probe_c * 1000.0 / R.probe_ms : 0.0;
    out->sched_tx_per_s = R.sched_ms > 0 ? R.sched_c * 1000.0 / R.sched_ms : 0.0;
    out->probe_abort_rate = R.probe_c + R.probe_a ? (double)R.probe_a / (double)(R.probe_c + R.probe_a) : 0.0;
    out->sched_abort_rate = R.sched_c + R.sched_a ? (double)R.sched_a / (double)(R.sched_c + R.sched_a) : 0.0;
    out->predict_ms = R.pred_ms;
    out->train_ms = R.train_ms;
    if (hc.err) return (int)hc.err;
    if (hc.committed != n) return GCC_ESTATE;
    return GCC_OK;
}

}  // namespace

extern "C" {

int gcc_sched_run(gcc_sched *sc, const gcc_run_params *rp, gcc_sched_result *out) {
    cudaGetLastError();
    if (!sc || !rp || !out) return GCC_EINVAL;
    memset(out, 0, sizeof(*out));
    gcc_engine *e = sc->e;
    if (!e->txs || e->n_rec == 0) return GCC_ESTATE;
    if (rp->batch_size < 1 || rp->batch_size > (1 << 20)) return GCC_EINVAL;
    const uint64_t n = e->n_rec;
    const uint64_t batch = std::min<uint64_t>((uint64_t)rp->batch_size, n);
    const uint64_t nb = (n + batch - 1) / batch;
    SchedRun R;
    int rc = sched_setup(R, sc, rp, false, batch);
    if (rc) return rc;
    sc->batches.assign(nb, gcc_sched_batch{});
    for (uint64_t b = 0; b < nb; ++b) {
        const uint64_t bst = b * batch, bn = std::min<uint64_t>(batch, n - bst);
        rc = sched_batch(R, bst, bn, sc->batches[b]);
        if (rc) break;
    }
    const int rc2 = sched_finish(R, n, nb, out);
    return rc ? rc : rc2;
}

int gcc_serve(gcc_sched *sc, const gcc_run_params *rp, const gcc_serve_params *sp,
              gcc_serve_result *out) {
    cudaGetLastError();
    if (!sc || !rp || !sp || !out) return GCC_EINVAL;
    memset(out, 0, sizeof(*out));
    gcc_engine *e = sc->e;
    if (!e->n_var || !e->reqs_d) return GCC_ESTATE;
    if (!(sp->rate_tps > 0.0) || sp->max_batch < 0 || sp->min_batch < 0 || !(sp->max_wait_us >= 0.0))
        return GCC_EINVAL;
    const uint64_t n = e->n_var;
    cudaSetDevice(e->dev);
    // admission cap: the caller's, else what half the free device memory
    // holds at the scheduler's per-transaction footprint (activations,
    // features, probabilities, labels, partition scratch)
    uint64_t cap = sp->max_batch ? (uint64_t)sp->max_batch : 0;
    if (!cap) {
        size_t fr = 0, tot = 0;
        cudaError_t ce = cudaMemGetInfo(&fr, &tot);
        if (ce != cudaSuccess) return e->fail_cuda(ce);
        const uint64_t per_tx = 4ull * sched::kHid * 4 + sched::kFeatStride * 2 + 16;
        cap = (uint64_t)(fr / 2) / per_tx;
    }
    cap = std::max<uint64_t>(1, std::min<uint64_t>({cap, 1ull << 20, n}));
    SchedRun R;
    int rc = sched_setup(R, sc, rp, true, cap);
    if (rc) return rc;
    // Poisson arrivals: exponential gaps from a counter-based hash
    std::vector<double> arrive(n);
    double t = 0.0;
    for (uint64_t i = 0; i < n; ++i) {
        const double u = ((double)(hash3(sp->seed, i, 0x415252ull) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
        t += -std::log(u) / sp->rate_tps;
        arrive[i] = t;
    }
    const uint64_t min_b = sp->min_batch ? (uint64_t)sp->min_batch : 1;
    const double max_wait = (sp->max_wait_us > 0.0 ? sp->max_wait_us : 200.0) * 1e-6;
    std::vector<double> lat(n);
    sc->batches.clear();
    const auto t0 = std::chrono::steady_clock::now();
    auto now = [&]() { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); };
    uint64_t next = 0, arrived = 0;
    double busy = 0.0;
    while (next < n) {
        const double tn = now();
        while (arrived < n && arrive[arrived] <= tn) ++arrived;
        const uint64_t waiting = arrived - next;
        if (waiting == 0 || (waiting < min_b && tn - arrive[next] < max_wait && arrived < n)) {
            // idle until the next arrival (or the wait bound), sleeping when
            // that is far enough away
            const double until = waiting == 0 ? arrive[next] : arrive[next] + max_wait;
            const double dt = until - tn;
            if (dt > 200e-6)
                std::this_thread::sleep_for(std::chrono::microseconds((int64_t)((dt - 100e-6) * 1e6)));
            continue;
        }
        const uint64_t bn = std::min<uint64_t>(waiting, cap);
        sc->batches.push_back(gcc_sched_batch{});
        const double b0 = now();
        rc = sched_batch(R, next, bn, sc->batches.back());
        const double b1 = now();
        busy += b1 - b0;
        if (rc) break;
        for (uint64_t i = next; i < next + bn; ++i) lat[i] = b1 - arrive[i];
        next += bn;
    }
    const double wall = now();
    gcc_sched_result sr;
    memset(&sr, 0, sizeof(sr));
    const int rc2 = sched_finish(R, rc ? next : n, sc->batches.size(), &sr);
    if (rc) return rc;
    if (rc2) return rc2;
    std::vector<double> ls(lat.begin(), lat.begin() + next);
    std::sort(ls.begin(), ls.end());
    auto q = [&](double f) {
        return ls.empty() ? 0.0 : ls[std::min<size_t>(ls.size() - 1, (size_t)(f * ls.size()))] * 1e6;
    };
    out->committed = sr.run.committed;
    out->aborts = sr.run.aborts;
    out->batches = sc->batches.size();
    out->admit_cap = cap;
    out->offered_tps = n / arrive[n - 1];
    out->tx_per_s = wall > 0 ? sr.run.committed / wall : 0.0;
    out->device_tx_per_s = sr.run.tx_per_s;
    out->lat_p50_us = q(0.50);
    out->lat_p99_us = q(0.99);
    out->lat_max_us = ls.empty() ? 0.0 : ls.back() * 1e6;
    out->mean_batch = out->batches ? (double)n / (double)out->batches : 0.0;
    out->busy_frac = wall > 0 ? busy / wall : 0.0;
    out->sched_abort_rate = sr.sched_abort_rate;
    out->kernel_launches = sr.run.kernel_launches;
    return GCC_OK;
}

}  // extern "C"
