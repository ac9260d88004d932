// gcc_common.cuh -- shared device-side definitions of the transaction engine:
// value formulas (table fill, field writes, read digests), packed metadata
// word formats, bounded waits, key -> row index probes and the kernel
// parameter block.
#pragma once
#include <stdint.h>
#include <cuda_runtime.h>
#include "../../include/gcc_engine.h"

#define GCC_HD __host__ __device__ __forceinline__
#define GCC_D __device__ __forceinline__

namespace gcc {

constexpr int kMaxOps = 16;              // requests per gen_ycsb record
constexpr int kMaxVarOps = 64;           // requests per variable-length transaction
constexpr uint32_t kNoRow = 0xFFFFFFFFu; // index miss / padding op
constexpr uint64_t kGolden = 0x9E3779B97F4A7C15ull;

// ---------------------------------------------------------------------------
// Value formulas. The CPU oracle restates these independently.
// ---------------------------------------------------------------------------
GCC_HD uint64_t splitmix64(uint64_t x) {
    uint64_t z = x + kGolden;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
// Keyed hash of two counters.
GCC_HD uint64_t hash3(uint64_t s, uint64_t a, uint64_t b) {
    return splitmix64(splitmix64(s ^ (a * kGolden)) ^ (b * 0xC2B2AE3D27D4EB4Full));
}
// Word k of row r after table initialisation (before the key / id is put in).
GCC_HD uint64_t fill_word(uint64_t seed, uint64_t row, uint32_t k) {
    return seed ? hash3(seed, row, k) : 0ull;
}
// GCC_WRITE_FIELD: field index in [0,10) and value of op i of transaction tx.
GCC_HD uint32_t write_field(uint64_t wseed, uint64_t tx, uint32_t i) {
    return (uint32_t)(hash3(wseed, tx, 2ull * i) % 10ull);
}
GCC_HD uint64_t write_value(uint64_t wseed, uint64_t tx, uint32_t i) {
    return hash3(wseed, tx, 2ull * i + 1ull);
}
// Read digest: sum over read ops i and row words k of mix(word, i, k), so the
// lanes of a transaction can add their parts in any order.
GCC_HD uint64_t digest_term(uint64_t word, uint32_t i, uint32_t k) {
    return splitmix64(word ^ ((uint64_t)(i * 16u + k + 1u) * 0xD6E8FEB86659FD93ull));
}

// ---------------------------------------------------------------------------
// Packed 64-bit metadata words (one per row, separate array, L2 friendly).
// ---------------------------------------------------------------------------
// 2PL: bits 0..30 shared-holder count, bit 31 exclusive, bits 32..62 holder
// (the exclusive holder's transaction id; wait-die compares it).
namespace tpl {
constexpr uint64_t kReaders = 0x7FFFFFFFull;
constexpr uint64_t kExcl = 1ull << 31;
GCC_HD uint64_t excl_word(uint32_t tx) { return kExcl | ((uint64_t)tx << 32); }
GCC_HD uint32_t holder(uint64_t w) { return (uint32_t)(w >> 32) & 0x7FFFFFFFu; }
}  // namespace tpl
// TO / MVCC: bit 63 uncommitted, bits 31..61 rts, bits 0..30 wts (31-bit
// timestamps as in the reference's {uncommited:1, rts:31, wts:31}).
namespace tso {
constexpr uint64_t kUnc = 1ull << 63;
constexpr uint64_t kTsMax = (1ull << 31) - 1;
GCC_HD uint64_t wts(uint64_t w) { return w & kTsMax; }
GCC_HD uint64_t rts(uint64_t w) { return (w >> 31) & kTsMax; }
GCC_HD uint64_t make(bool unc, uint64_t rts, uint64_t wts) {
    return (unc ? kUnc : 0ull) | (rts << 31) | wts;
}
}  // namespace tso
// Silo: bit 63 lock, bits 0..62 tid/timestamp.
namespace silo {
constexpr uint64_t kLock = 1ull << 63;
GCC_HD uint64_t ts(uint64_t w) { return w & ~kLock; }
}  // namespace silo
// TicToc: bit 63 lock, bits 48..62 delta (rts - wts), bits 0..47 wts.
namespace tictoc {
constexpr uint64_t kLock = 1ull << 63;
constexpr uint64_t kWtsMask = (1ull << 48) - 1;
GCC_HD uint64_t wts(uint64_t w) { return w & kWtsMask; }
GCC_HD uint64_t delta(uint64_t w) { return (w >> 48) & 0x7FFFull; }
GCC_HD uint64_t rts(uint64_t w) { return wts(w) + delta(w); }
GCC_HD uint64_t make(bool lock, uint64_t delta, uint64_t wts) {
    return (lock ? kLock : 0ull) | (delta << 48) | (wts & kWtsMask);
}
}  // namespace tictoc

// ---------------------------------------------------------------------------
// Run-wide counters, metrics and latency histogram (device memory).
// ---------------------------------------------------------------------------
constexpr int kHistBuckets = 1024;  // 64 octaves x 16 linear sub-buckets (ns)
constexpr int kTicketStripes = 32;  // ticket counters, one per 128-byte line

struct Counters {
    // stripe j hands out positions j, j + 32, j + 64, ... in order
    unsigned long long tickets[kTicketStripes * 16];
    unsigned long long seq;        // serialization sequence (commit log)
    unsigned long long ts;         // timestamp allocator (TO, MVCC)
    unsigned long long committed;  // committed transactions
    unsigned long long aborts;     // aborted attempts
    unsigned long long ts_cycles, wait_cycles, abort_cycles, mng_cycles,
        tot_cycles, idx_cycles;    // clock64 sums (reference Metrics)
    unsigned long long max_rank;   // gputx
    unsigned int err;              // first error status (negative gcc code)
    unsigned int err_where;        // diagnostic: which wait gave up
    unsigned int max_attempts;     // most attempts of one transaction
    unsigned int starving;         // transactions past the starvation limit
    unsigned int starve_token;     // 0, or 1 + tx of the starving tx that retries
    unsigned int hist[kHistBuckets];
};

GCC_HD uint32_t hist_bucket(uint64_t ns) {
    if (ns < 16) return (uint32_t)ns;
#ifdef __CUDA_ARCH__
    uint32_t lg = 63u - (uint32_t)__clzll((long long)ns);  // >= 4
#else
    uint32_t lg = 63u - (uint32_t)__builtin_clzll(ns);  // >= 4
#endif
    uint32_t sub = (uint32_t)((ns >> (lg - 4)) & 15u);
    uint32_t b = (lg - 3u) * 16u + sub;
    return b < (uint32_t)kHistBuckets ? b : (uint32_t)kHistBuckets - 1u;
}

// ---------------------------------------------------------------------------
// Kernel parameter block.
// ---------------------------------------------------------------------------
struct KParams {
    const gcc_ycsb_tx *txs;     // all loaded transactions (16-request records)
    const uint32_t *tx_off;     // variable-length transactions: requests of tx t
    const gcc_ycsb_req *reqs;   //   are reqs[tx_off[t] .. tx_off[t+1]) (else null)
    uint32_t n_tx;              // loaded transactions
    uint32_t slot_ops;          // request slots per position / tx (16 or 64)
    uint32_t batch_st;          // first position of this launch
    uint32_t batch_n;           // positions in this launch
    const volatile unsigned long long *queue_tail;  // admitted positions (device
                                // queue; null: all batch_n are admitted)
    const uint32_t *order;      // position -> tx id (null: batch_st + pos)
    // index
    int32_t index_kind;
    const unsigned long long *hash_slots;  // {key | row << 32}, 4 per bucket
    uint64_t hash_bucket_mask;
    const unsigned long long *sorted;      // {key | row << 32} sorted by key
    uint32_t sorted_len;
    uint64_t rows;
    // table
    uint8_t *table;
    uint32_t stride;            // bytes between rows (16-byte multiple)
    uint32_t words;             // 8-byte words of row payload (11 or 13)
    uint32_t wslot;             // words per row image slot (words rounded to even)
    int32_t write_mode;
    uint64_t write_seed;
    // CC metadata
    unsigned long long *meta;   // one packed word per row
    unsigned int *latch;        // per-row latch (slow_* schemes)
    unsigned int *turn;         // per-row turn (gacco/gputx) / mvcc chain head
    // MVCC version store: one node per (batch position, op)
    unsigned long long *ver_ts;   // old version word
    unsigned int *ver_prev;       // previous node or kNoRow
    uint64_t *ver_data;           // old row image (wslot words per node)
    // precomputed per access (ordered schemes): access = pos * 16 + op
    const uint32_t *op_row;
    const uint32_t *op_pos;
    // outputs, indexed by tx id
    unsigned long long *digest;
    unsigned long long *commit_hi;
    unsigned long long *commit_lo;
    unsigned int *tx_aborts;
    uint64_t *read_log;         // (tx * 16 + op) * wslot, or null
    uint64_t *scratch;          // rowcopy buffers, (pos * 16 + op) * wslot
    Counters *ctr;
    uint64_t spin_limit_ns;
    uint32_t flags;
    uint32_t wait_die;
    uint32_t backoff_ns;        // 0: retry at once
    uint32_t starve_limit;      // 0: no starvation control
    uint32_t ext_ops;           // the loaded transactions hold extended ops
    // 2PL lock plan of each transaction (indexed by tx id, 16-request
    // records only; null: none). Bits 0-15 mark the requests locked after
    // the others, one at a time; bits 16-19 count them (<= kPlanMax) and
    // nibble j at bit 20 + 4j is the request index of the j-th of them.
    const unsigned long long *plan;
    uint32_t ordered_from;      // attempts from which 2PL / TO visit one request
                                // at a time: 0 = the scheme's default, k = k - 1
};

constexpr int kPlanMax = 11;  // planned requests that fit the nibble list
GCC_HD uint32_t plan_mask(unsigned long long pl) { return (uint32_t)(pl & 0xFFFFull); }
GCC_HD uint32_t plan_count(unsigned long long pl) { return (uint32_t)((pl >> 16) & 0xFull); }
GCC_HD uint32_t plan_op(unsigned long long pl, uint32_t j) { return (uint32_t)((pl >> (20 + 4 * j)) & 0xFull); }

// ---------------------------------------------------------------------------
// Small device helpers.
// ---------------------------------------------------------------------------
GCC_D uint64_t gtimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
GCC_D unsigned long long ld_cg(const unsigned long long *p) {
    return __ldcg(p);
}
GCC_D unsigned int ld_cg(const unsigned int *p) { return __ldcg(p); }
GCC_D unsigned long long ld_volatile(const unsigned long long *p) {
    return *(const volatile unsigned long long *)p;
}
GCC_D unsigned int ld_volatile(const unsigned int *p) {
    return *(const volatile unsigned int *)p;
}
// Acquire/release fence at GPU scope: orders this thread's earlier memory
// operations before its later ones, which is all the lock/timestamp
// protocols here need (no store->load Dekker patterns), and is cheaper than
// the sequentially consistent fence behind __threadfence().
GCC_D void fence_acq_rel() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

// Atomics with acquire / release semantics at GPU scope: the lock RMW orders
// this lane's later accesses to the row after it (acquire) and the unlock
// RMW orders its earlier accesses before it (release), without a standalone
// fence.
GCC_D unsigned long long atom_add_acq(unsigned long long *p, unsigned long long v) {
    unsigned long long r;
    asm volatile("atom.acquire.gpu.global.add.u64 %0, [%1], %2;" : "=l"(r) : "l"(p), "l"(v) : "memory");
    return r;
}
GCC_D unsigned long long atom_cas_acq(unsigned long long *p, unsigned long long cmp,
                                      unsigned long long val) {
    unsigned long long r;
    asm volatile("atom.acquire.gpu.global.cas.b64 %0, [%1], %2, %3;"
                 : "=l"(r) : "l"(p), "l"(cmp), "l"(val) : "memory");
    return r;
}
GCC_D void red_add_rel(unsigned long long *p, unsigned long long v) {
    asm volatile("red.release.gpu.global.add.u64 [%0], %1;" :: "l"(p), "l"(v) : "memory");
}
GCC_D void red_and_rel(unsigned long long *p, unsigned long long v) {
    asm volatile("red.release.gpu.global.and.b64 [%0], %1;" :: "l"(p), "l"(v) : "memory");
}
GCC_D unsigned ld_acquire(const unsigned *p) {
    unsigned r;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(r) : "l"(p) : "memory");
    return r;
}
GCC_D void st_release(unsigned *p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" :: "l"(p), "r"(v) : "memory");
}

GCC_D void set_error(Counters *c, int code, unsigned where) {
    if (atomicCAS(&c->err, 0u, (unsigned)code) == 0u) c->err_where = where;
}
GCC_D bool error_raised(const Counters *c) {
    return *(const volatile unsigned int *)&c->err != 0u;
}

// Row access: payload words as 8-byte words; rows are 16-byte aligned.
GCC_D uint64_t *row_ptr(const KParams &p, uint32_t row) {
    return (uint64_t *)(p.table + (size_t)row * p.stride);
}

// Load the whole row payload with 16-byte L2 loads (bypassing L1 so that
// writes by other SMs are seen). `w` receives p.words words.
template <int MAXW>
GCC_D void load_row(const KParams &p, uint32_t row, uint64_t (&w)[MAXW]) {
    const ulonglong2 *src = (const ulonglong2 *)row_ptr(p, row);
#pragma unroll
    for (int c = 0; c < MAXW / 2; ++c) {
        if (2 * c < (int)p.words) {
            ulonglong2 v = __ldcg(src + c);
            w[2 * c] = v.x;
            w[2 * c + 1] = v.y;
        }
    }
}

// ---------------------------------------------------------------------------
// Index probes (all keys are 32-bit, like SortedArray_GPU<unsigned int>).
// ---------------------------------------------------------------------------
GCC_HD uint64_t hash_bucket_of(uint32_t key, uint64_t mask) {
    return splitmix64((uint64_t)key) & mask;
}

// Returns the row of `key` or kNoRow. Hash buckets are one 32-byte DRAM
// sector (4 slots of {key, row}); a probe reads one sector with two 16-byte
// loads, linear probing on overflow.
GCC_D uint32_t index_find(const KParams &p, uint32_t key) {
    if (p.index_kind == GCC_INDEX_DIRECT) {
        return (uint64_t)key < p.rows ? key : kNoRow;
    }
    if (p.index_kind == GCC_INDEX_HASH) {
        uint64_t b = hash_bucket_of(key, p.hash_bucket_mask);
        for (uint64_t probe = 0; probe <= p.hash_bucket_mask; ++probe) {
            const ulonglong2 *bk = (const ulonglong2 *)(p.hash_slots + 4 * b);
            ulonglong2 s01 = __ldg(bk);
            ulonglong2 s23 = __ldg(bk + 1);
            unsigned long long s[4] = {s01.x, s01.y, s23.x, s23.y};
            bool empty = false;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if (s[j] == ~0ull) { empty = true; continue; }
                if ((uint32_t)s[j] == key) return (uint32_t)(s[j] >> 32);
            }
            if (empty) return kNoRow;
            b = (b + 1) & p.hash_bucket_mask;
        }
        return kNoRow;
    }
    // GCC_INDEX_SORTED: binary search of SortedArray_GPU::Find
    // (include/index.cuh:74-91); a miss returns kNoRow instead of `length`.
    uint32_t st = 0, en = p.sorted_len;
    while (st < en) {
        uint32_t mid = (st + en) >> 1;
        unsigned long long it = __ldg(p.sorted + mid);
        uint32_t k = (uint32_t)it;
        if (k == key) return (uint32_t)(it >> 32);
        if (k > key) en = mid; else st = mid + 1;
    }
    return kNoRow;
}

}  // namespace gcc
