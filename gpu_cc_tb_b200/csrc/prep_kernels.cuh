// prep_kernels.cuh -- device passes that run around the transaction kernel:
// table fill, index build, a stable LSD radix sort of (u32 key, u32 value)
// pairs, a multi-level prefix scan, and the ordering passes of GaccO and
// GPUTx.
//
// Reference behaviour followed:
//   GaccO per-batch precompute      include/gacco.cuh:244-339, src/gacco.cu:5-15
//     (count per object, dense ids, thrust sort_by_key/exclusive_scan/sort of
//      (obj, tx) pairs, then aux[obj] = {offset, lock = first tx})
//   GPUTx ranking                   include/gputx.cuh:213-299, src/gputx.cu:5-38
//     (rank of an access = number of read/write or write/write boundaries
//      before it in its object's tx-ordered list; tx rank = max over its
//      accesses; txs grouped by rank)
// Here both become: one stable sort of access keys by row, then flat
// per-position passes (no per-object serial walk, no host round trip).
#pragma once
#include "gcc_common.cuh"

namespace gcc {

// ---------------------------------------------------------------------------
// Table fill and index build.
// ---------------------------------------------------------------------------
// Row r: word 0 carries the key (u64x11: uint64 key = r; ref104: uint32 id = r
// in the low half, random bytes above), words 1.. are fill_word(seed, r, k).
__global__ void k_fill_table(uint8_t *table, uint64_t rows, uint32_t stride, uint32_t words,
                             int32_t layout, uint64_t seed) {
    uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (r >= rows) return;
    uint64_t *w = (uint64_t *)(table + r * stride);
    uint32_t slot = stride / 8;
    for (uint32_t k = 0; k < slot; ++k) {
        uint64_t v = 0;
        if (k < words) {
            v = fill_word(seed, r, k);
            if (k == 0) v = (layout == GCC_LAYOUT_U64X11) ? r : ((v & 0xFFFFFFFF00000000ull) | (uint32_t)r);
        }
        w[k] = v;
    }
}

__device__ __forceinline__ uint32_t row_key(const uint8_t *table, uint64_t r, uint32_t stride) {
    return (uint32_t)(*(const uint64_t *)(table + r * stride));
}

// Insert (key of row r, r) into the bucketed hash table (4 slots / bucket).
__global__ void k_hash_insert(const uint8_t *table, uint64_t rows, uint32_t stride,
                              unsigned long long *slots, uint64_t bucket_mask, unsigned *err) {
    uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (r >= rows) return;
    uint32_t key = row_key(table, r, stride);
    unsigned long long ent = (unsigned long long)key | ((unsigned long long)r << 32);
    uint64_t b = hash_bucket_of(key, bucket_mask);
    for (uint64_t probe = 0; probe <= bucket_mask; ++probe) {
        for (int j = 0; j < 4; ++j) {
            unsigned long long old = atomicCAS(slots + 4 * b + j, ~0ull, ent);
            if (old == ~0ull) return;
        }
        b = (b + 1) & bucket_mask;
    }
    atomicCAS(err, 0u, (unsigned)GCC_ENOMEM);
}

__global__ void k_sorted_entries(const uint8_t *table, uint64_t rows, uint32_t stride,
                                 uint32_t *keys, uint32_t *vals) {
    uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (r >= rows) return;
    keys[r] = row_key(table, r, stride);
    vals[r] = (uint32_t)r;
}
__global__ void k_pack_sorted(const uint32_t *keys, const uint32_t *vals, uint64_t n,
                              unsigned long long *out) {
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = (unsigned long long)keys[i] | ((unsigned long long)vals[i] << 32);
}

__global__ void k_index_lookup(KParams p, const uint32_t *keys, uint32_t *rows, uint64_t n) {
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    rows[i] = index_find(p, keys[i]);
}

// ---------------------------------------------------------------------------
// Prefix scan of u32 (exclusive or inclusive), 4096 items per block.
// ---------------------------------------------------------------------------
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t *warp_sums,
                                                         uint32_t &total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[wid] = x;
    __syncthreads();
    if (wid == 0) {
        uint32_t s = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xFFFFFFFFu, s, o);
            if (lane >= o) s += y;
        }
        warp_sums[lane] = s;  // inclusive per warp
    }
    __syncthreads();
    uint32_t warp_base = wid ? warp_sums[wid - 1] : 0u;
    total = warp_sums[(blockDim.x >> 5) - 1];
    __syncthreads();
    return warp_base + x - v;
}

// Scan `in` (n items) into `out`; per-block totals to `sums` (may be null).
__global__ void __launch_bounds__(kScanThreads) k_scan_tile(const uint32_t *in, uint32_t *out,
                                                            uint64_t n, uint32_t *sums,
                                                            int inclusive) {
    __shared__ uint32_t warp_sums[32];
    const uint64_t base = (uint64_t)blockIdx.x * kScanTile + (uint64_t)threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t t = 0;
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        v[j] = (base + j < n) ? in[base + j] : 0u;
        t += v[j];
    }
    uint32_t total;
    uint32_t ex = block_exclusive_scan(t, warp_sums, total);
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        uint32_t o = inclusive ? ex + v[j] : ex;
        if (base + j < n) out[base + j] = o;
        ex += v[j];
    }
    if (sums && threadIdx.x == 0) sums[blockIdx.x] = total;
}
__global__ void k_scan_add(uint32_t *out, uint64_t n, const uint32_t *block_prefix) {
    uint64_t i = blockIdx.x * (uint64_t)kScanTile + threadIdx.x;
    uint32_t add = block_prefix[blockIdx.x];
    for (int j = 0; j < kScanItems; ++j, i += kScanThreads)
        if (i < n) out[i] += add;
}

// ---------------------------------------------------------------------------
// Stable LSD radix sort, 8-bit digits, 4096 items per block.
// counts are digit-major: counts[d * nblocks + b].
// ---------------------------------------------------------------------------
constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortRounds = 16;                       // per warp
constexpr int kSortTile = kSortThreads * kSortRounds;  // 4096
constexpr int kRadix = 256;

__global__ void __launch_bounds__(kSortThreads) k_sort_hist(const uint32_t *keys, uint64_t n,
                                                            int shift, uint32_t *counts,
                                                            uint32_t nblocks) {
    __shared__ uint32_t h[kRadix];
    for (int i = threadIdx.x; i < kRadix; i += kSortThreads) h[i] = 0;
    __syncthreads();
    const uint64_t base = (uint64_t)blockIdx.x * kSortTile;
    for (int j = 0; j < kSortRounds; ++j) {
        uint64_t i = base + (uint64_t)j * kSortThreads + threadIdx.x;
        if (i < n) atomicAdd(&h[(keys[i] >> shift) & 0xFFu], 1u);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < kRadix; d += kSortThreads)
        counts[(uint64_t)d * nblocks + blockIdx.x] = h[d];
}

// Each warp owns a contiguous 512-item slice of the tile (rounds of 32), so
// (warp, round, lane) order is input order and ranks are stable.
__global__ void __launch_bounds__(kSortThreads) k_sort_scatter(
    const uint32_t *keys_in, const uint32_t *vals_in, uint64_t n, int shift,
    const uint32_t *offsets, uint32_t nblocks, uint32_t *keys_out, uint32_t *vals_out) {
    __shared__ uint32_t wcnt[kSortWarps][kRadix];
    __shared__ uint32_t dbase[kRadix];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < kSortWarps * kRadix; i += kSortThreads) (&wcnt[0][0])[i] = 0;
    __syncthreads();
    const uint64_t base = (uint64_t)blockIdx.x * kSortTile + (uint64_t)wid * (32 * kSortRounds);
    uint32_t k[kSortRounds], rk[kSortRounds];
    const unsigned lt = (1u << lane) - 1u;
#pragma unroll
    for (int r = 0; r < kSortRounds; ++r) {
        uint64_t i = base + (uint64_t)r * 32 + lane;
        bool ok = i < n;
        k[r] = ok ? keys_in[i] : 0u;
        uint32_t d = ok ? ((k[r] >> shift) & 0xFFu) : 0x100u;
        unsigned peers = __match_any_sync(0xFFFFFFFFu, d);
        uint32_t before = ok ? wcnt[wid][d] : 0u;
        rk[r] = before + __popc(peers & lt);
        __syncwarp();
        if (ok && (peers & lt) == 0u) wcnt[wid][d] = before + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    for (int d = threadIdx.x; d < kRadix; d += kSortThreads) {
        uint32_t run = offsets[(uint64_t)d * nblocks + blockIdx.x];
        dbase[d] = run;
        for (int w = 0; w < kSortWarps; ++w) {
            uint32_t c = wcnt[w][d];
            wcnt[w][d] = run;
            run += c;
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kSortRounds; ++r) {
        uint64_t i = base + (uint64_t)r * 32 + lane;
        if (i < n) {
            uint32_t d = (k[r] >> shift) & 0xFFu;
            uint32_t dst = wcnt[wid][d] + rk[r];
            keys_out[dst] = k[r];
            vals_out[dst] = vals_in[i];
        }
    }
}

// ---------------------------------------------------------------------------
// Access lists of the ordered schemes. Access a = pos * 16 + op.
// ---------------------------------------------------------------------------
// key = row (or `invalid_key` for padding ops so they sort last),
// val = a | read << 31. op_row[a] = row or kNoRow.
__global__ void k_access_build(KParams p, uint64_t n_pos, uint32_t invalid_key, uint32_t *keys,
                               uint32_t *vals, uint32_t *op_row) {
    uint64_t a = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (a >= n_pos * kMaxOps) return;
    uint64_t pos = a / kMaxOps;
    uint32_t i = (uint32_t)(a % kMaxOps);
    uint32_t tx = p.order ? p.order[p.batch_st + pos] : p.batch_st + (uint32_t)pos;
    const gcc_ycsb_tx *T = p.txs + tx;
    uint64_t n = T->request_cnt;
    uint32_t row = kNoRow, key = invalid_key, rd = 0;
    if (n > (uint64_t)kMaxOps) {
        if (i == 0) atomicCAS(&p.ctr->err, 0u, (unsigned)GCC_EFORMAT);
    } else if (i < n) {
        int2 rq = *(const int2 *)&T->requests[i];
        row = index_find(p, (uint32_t)rq.y);
        if (row == kNoRow) atomicCAS(&p.ctr->err, 0u, (unsigned)GCC_EKEY);
        else key = row;
        rd = rq.x > 0 ? 1u : 0u;
    }
    keys[a] = key;
    vals[a] = (uint32_t)a | (rd << 31);
    op_row[a] = row;
}

// After the stable sort by row: op_pos[a] = sorted position; the first
// position of each row's run becomes that row's initial turn.
__global__ void k_access_positions(const uint32_t *skeys, const uint32_t *svals, uint64_t n_acc,
                                   uint32_t invalid_key, uint32_t *op_pos, unsigned *turn) {
    uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (q >= n_acc) return;
    uint32_t row = skeys[q];
    if (row == invalid_key) return;
    op_pos[svals[q] & 0x7FFFFFFFu] = (uint32_t)q;
    if (q == 0 || skeys[q - 1] != row) turn[row] = (uint32_t)q;
}

// GPUTx: f[q] = 1 where a run continues and the pair (q-1, q) is not
// read/read (src/gputx.cu:24-25).
__global__ void k_rank_flags(const uint32_t *skeys, const uint32_t *svals, uint64_t n_acc,
                             uint32_t invalid_key, uint32_t *f) {
    uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (q >= n_acc) return;
    uint32_t row = skeys[q];
    uint32_t v = 0;
    if (row != invalid_key && q > 0 && skeys[q - 1] == row) {
        bool r0 = svals[q - 1] >> 31, r1 = svals[q] >> 31;
        v = (r0 && r1) ? 0u : 1u;
    }
    f[q] = v;
}
__global__ void k_rank_segbase(const uint32_t *skeys, const uint32_t *S, uint64_t n_acc,
                               uint32_t invalid_key, unsigned *segbase) {
    uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (q >= n_acc) return;
    uint32_t row = skeys[q];
    if (row == invalid_key) return;
    if (q == 0 || skeys[q - 1] != row) segbase[row] = S[q];
}
__global__ void k_rank_tx(const uint32_t *skeys, const uint32_t *svals, const uint32_t *S,
                          uint64_t n_acc, uint32_t invalid_key, const unsigned *segbase,
                          unsigned *tx_rank, unsigned long long *max_rank) {
    uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (q >= n_acc) return;
    uint32_t row = skeys[q];
    if (row == invalid_key) return;
    uint32_t r = S[q] - segbase[row];
    uint32_t tx = (svals[q] & 0x7FFFFFFFu) / kMaxOps;
    atomicMax(tx_rank + tx, r);
    atomicMax(max_rank, (unsigned long long)r);
}
__global__ void k_iota(uint32_t *v, uint64_t n) {
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i < n) v[i] = (uint32_t)i;
}

// Count differing 8-byte words of two buffers (replay check).
__global__ void k_count_diff(const unsigned long long *a, const unsigned long long *b, uint64_t n,
                             unsigned long long *diff) {
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    unsigned long long d = 0;
    for (; i < n; i += (uint64_t)gridDim.x * blockDim.x) d += a[i] != b[i];
    if (d) atomicAdd(diff, d);
}

// Device-side time stamp (%globaltimer, ns) into slots[i]: timing that also
// works inside a captured CUDA graph.
__global__ void k_stamp(unsigned long long *slots, int i) {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    slots[i] = t;
}

// Per-launch counter reset: ticket stripes = 0 and, for TO/MVCC, ts = 1
// (NaiveTSAllocator_CPU::Init, include/timestamp.cuh:76-80).
__global__ void k_batch_prep(Counters *c, int reset_ts) {
    if (threadIdx.x < kTicketStripes) c->tickets[threadIdx.x * 16] = 0ull;
    if (threadIdx.x == 0 && reset_ts) c->ts = 1ull;
}

}  // namespace gcc
