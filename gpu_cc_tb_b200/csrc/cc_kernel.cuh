// cc_kernel.cuh -- the YCSB transaction kernel under each concurrency-control
// scheme, written for sm_100a.
//
// Reference behaviour followed (gCCTB paths):
//   transaction loop + retry          benchmark/ycsb.cu:21-111
//   2PL no-wait / wait-die             include/twopl.cuh:59-382
//   timestamp ordering                 include/to.cuh:57-271
//   MVCC                               include/mvcc.cuh:61-297
//   Silo                               include/silo.cuh:70-339
//   TicToc                             include/tictoc.cuh:67-369
//   GaccO ordered hand-off             include/gacco.cuh:49-176
//   GPUTx rank execution               include/gputx.cuh:58-146
//   latch ("slow_") variants           include/slow_*.cuh, runtime.cuh:91-109
//
// B200 design (not a translation of the reference):
//   * persistent CTAs; a group of G = 2^warp_density lanes owns one
//     transaction at a time and takes the next from an ordered ticket;
//   * the G lanes split the transaction's requests: op i belongs to lane
//     i % G, so index probes, lock/timestamp operations and row copies of
//     different requests are in flight together (the reference runs them one
//     by one on lane 0); group-wide decisions are ballots;
//   * rows move with 16-byte L2 loads/stores (rows are 16-byte aligned);
//   * every wait is bounded by `spin_limit_ns` of %globaltimer and raises
//     GCC_ETIMEOUT instead of hanging.
//
// Commit rules are the reference's. Differences that fix reference bugs are
// listed where they occur (Silo commit timestamp, MVCC base-row update and
// version-store stride, GPUTx same-rank conflicts).
#pragma once
#include <cooperative_groups.h>
#include "gcc_common.cuh"

namespace gcc {

namespace cg = cooperative_groups;


enum Scheme : int {
    S_TPL_NW = 0, S_TPL_WD, S_TO, S_MVCC, S_SILO, S_TICTOC, S_GACCO, S_GPUTX,
    S_SLOW_TPL_NW, S_SLOW_TPL_WD, S_SLOW_TO, S_SLOW_MVCC, S_SLOW_SILO,
    S_SLOW_TICTOC, S_COUNT
};

enum AttemptStatus : int { kCommit = 0, kAbort = 1, kGiveUp = 2 };

// Where a bounded wait gave up (Counters::err_where).
enum WaitSite : unsigned {
    W_LATCH = 1, W_TPL_WD, W_TO_READ, W_MVCC_READ, W_SILO_READ, W_TICTOC_READ,
    W_TICTOC_EXT, W_TURN, W_RETRY, W_CAS, W_QUEUE, W_STARVE
};

// ---------------------------------------------------------------------------
// A group of G lanes of one warp working on one transaction.
// ---------------------------------------------------------------------------
template <int G>
struct Group {
    unsigned mask;  // lanes of this group within the warp
    int base;       // first lane of the group
    int glane;      // lane within the group
    GCC_D Group() {
        int lane = threadIdx.x & 31;
        base = lane & ~(G - 1);
        glane = lane & (G - 1);
        mask = (G == 32) ? 0xFFFFFFFFu : (((1u << G) - 1u) << base);
    }
    GCC_D bool any(bool p) const { return __any_sync(mask, p); }
    GCC_D void sync() const { __syncwarp(mask); }
    template <class T>
    GCC_D T bcast(T v, int src) const { return __shfl_sync(mask, v, src, G); }
    GCC_D unsigned long long sum(unsigned long long v) const {
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o, G);
        return v;
    }
    GCC_D unsigned long long maxv(unsigned long long v) const {
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) {
            unsigned long long u = __shfl_xor_sync(mask, v, o, G);
            v = u > v ? u : v;
        }
        return v;
    }
    GCC_D unsigned long long orv(unsigned long long v) const {
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) v |= __shfl_xor_sync(mask, v, o, G);
        return v;
    }
};

// Per-transaction lane state: lane owns ops i = glane + k*G, k < K, of a
// transaction of at most MO requests.
template <int G_, int MO>
struct TxOps {
    static constexpr int G = G_;
    static constexpr int MAXOPS = MO;
    static constexpr int K = (MO + G - 1) / G;
    static constexpr bool kExt = MO > kMaxOps;  // extended ops (var-length only)
    uint32_t n;                // requests in the transaction
    uint32_t valid;            // bit k: op k exists
    uint32_t isread;           // bit k: op k reads
    unsigned long long readmask;  // group-wide: bit i set if op i reads
    uint32_t row[K];
    // 1 + the request that failed in the last aborted 2PL / TO attempt (0:
    // none); the next one-at-a-time attempt visits it after the others
    // (unless GCC_F_REQUEST_ORDER)
    mutable uint32_t obst_op;
};

// Bounded wait helper: true once `limit` ns have passed since `t0`.
GCC_D bool expired(uint64_t t0, uint64_t limit) { return gtimer() - t0 > limit; }
// Pause inside a wait loop so that diverged lanes of the same warp (another
// transaction's group, possibly the one being waited for) get issue slots.
GCC_D void wait_pause() { __nanosleep(20); }

// ---------------------------------------------------------------------------
// Row images: digest, read log, rowcopy scratch, writes.
// ---------------------------------------------------------------------------
constexpr int kMaxChunks = 7;  // 16-byte chunks cover up to 14 words (112 B)

GCC_D size_t slot_of(const KParams &p, uint64_t unit, uint32_t i) {
    return ((size_t)unit * p.slot_ops + i) * p.wslot;
}
// Stream a row image from `src` (16-byte L2 loads), folding its words into
// the digest term `dt` of op i and copying it to the rowcopy scratch slot and
// the read log when those exist. Nothing is held in registers beyond one
// chunk, so the transaction kernel fits 64 registers.
GCC_D void read_image(const KParams &p, const uint64_t *src, uint32_t tx, uint64_t pos,
                      uint32_t i, unsigned long long &dt) {
    const ulonglong2 *s = (const ulonglong2 *)src;
    ulonglong2 *sc = p.scratch ? (ulonglong2 *)(p.scratch + slot_of(p, pos, i)) : nullptr;
    ulonglong2 *lg = p.read_log ? (ulonglong2 *)(p.read_log + slot_of(p, tx, i)) : nullptr;
#pragma unroll
    for (int c = 0; c < kMaxChunks; ++c) {
        if (2 * c < (int)p.words) {
            ulonglong2 v = __ldcg(s + c);
            dt += digest_term(v.x, i, 2u * c);
            if (2 * c + 1 < (int)p.words) dt += digest_term(v.y, i, 2u * c + 1u);
            if (sc) __stcg(sc + c, v);
            if (lg) __stcg(lg + c, v);
        }
    }
}
GCC_D void copy_image(const KParams &p, uint64_t *dst, const uint64_t *src) {
#pragma unroll
    for (int c = 0; c < kMaxChunks; ++c)
        if (2 * c < (int)p.words)
            __stcg((ulonglong2 *)dst + c, __ldcg((const ulonglong2 *)src + c));
}
// Last read op before op i (program order), -1 if none.
GCC_D int rowcopy_src(unsigned long long readmask, uint32_t i) {
    unsigned long long m = readmask & ((1ull << i) - 1ull);
    return m ? 63 - __clzll((long long)m) : -1;
}
// Extended write op (a request whose `read` word is negative, see
// gcc_engine.h GCC_OP_*): an integer read-modify-write of row fields, or an
// insert of a fresh row. Runs with the row held exclusively by the
// transaction (2PL lock, OCC write lock at commit, TO uncommitted mark,
// ordered turn); read-modify-writes fold the row image they read into the
// digest like a read.
GCC_D unsigned long long apply_ext(const KParams &p, uint64_t *r, uint32_t tx, uint32_t i,
                                  uint32_t w) {
    const uint32_t op = (w >> 28) & 7u, f = (w >> 24) & 15u, v = w & 0xFFFFFFu;
    const uint32_t fmax = op == GCC_OP_STOCK ? 6u : (op == GCC_OP_PAY ? 7u : 9u);
    if (op < GCC_OP_ADD || op > GCC_OP_INSERT || f > fmax || p.words != 11u) {
        set_error(p.ctr, GCC_EFORMAT, 0);
        return 0ull;
    }
    if (op == GCC_OP_INSERT) {
        __stcg((unsigned long long *)(r + 1), (unsigned long long)tx);
        __stcg((unsigned long long *)(r + 2), (unsigned long long)v);
#pragma unroll
        for (uint32_t k = 0; k < 8; ++k)
            __stcg((unsigned long long *)(r + 3 + k),
                   (unsigned long long)hash3(p.write_seed, tx, 1024ull + i * 8ull + k));
        return 0ull;
    }
    unsigned long long dt = 0;
    read_image(p, r, tx, 0, i, dt);
    unsigned long long *fw = (unsigned long long *)(r + 1 + f);
    const unsigned long long a = __ldcg(fw);
    if (op == GCC_OP_ADD) {
        __stcg(fw, a + v);
    } else if (op == GCC_OP_SUB) {
        __stcg(fw, a - v);
    } else if (op == GCC_OP_STOCK) {
        const unsigned long long q = v & 0xFFu, remote = (v >> 8) & 1u;
        __stcg(fw, a >= q + 10u ? a - q : a - q + 91u);
        __stcg(fw + 1, __ldcg(fw + 1) + q);
        __stcg(fw + 2, __ldcg(fw + 2) + 1u);
        __stcg(fw + 3, __ldcg(fw + 3) + remote);
    } else if (op == GCC_OP_PAY) {
        __stcg(fw, a - v);
        __stcg(fw + 1, __ldcg(fw + 1) + v);
        __stcg(fw + 2, __ldcg(fw + 2) + 1u);
    }
    return dt;
}

// Apply write op i of tx to `row` (GCC_WRITE_FIELD or GCC_WRITE_ROWCOPY, or
// an extended op when the run enables them). Extended ops exist only in the
// variable-length kernels (EXT): the 16-request kernels keep their registers.
template <bool EXT>
GCC_D void apply_write(const KParams &p, uint32_t row, uint32_t tx, uint64_t pos,
                       uint32_t i, unsigned long long readmask, unsigned long long &dg) {
    uint64_t *r = row_ptr(p, row);
    if (EXT && p.ext_ops) {
        const int32_t w = p.txs ? __ldg(&p.txs[tx].requests[i].read)
                                : __ldg(&p.reqs[p.tx_off[tx] + i].read);
        if (w < 0) {
            dg += apply_ext(p, r, tx, i, (uint32_t)w);
            return;
        }
    }
    if (p.write_mode == GCC_WRITE_FIELD) {
        uint32_t f = write_field(p.write_seed, tx, i);
        __stcg((unsigned long long *)(r + 1 + f),
               (unsigned long long)write_value(p.write_seed, tx, i));
        return;
    }
    int src = rowcopy_src(readmask, i);
    if (src < 0) {
#pragma unroll
        for (int c = 0; c < kMaxChunks; ++c)
            if (2 * c < (int)p.words) __stcg((ulonglong2 *)r + c, make_ulonglong2(0ull, 0ull));
    } else {
        copy_image(p, r, p.scratch + slot_of(p, pos, (uint32_t)src));
    }
}

// ---------------------------------------------------------------------------
// Retry timing: after an aborted attempt has released everything it held,
// the lane whose request failed polls that row's word (plain loads, short
// sleeps) until it looks compatible, at most kObstacleWaitNs, so the retry
// is not spent against the same conflict. The lock requests themselves keep
// the scheme's rule (e.g. no-wait: a conflicting request aborts).
// ---------------------------------------------------------------------------
constexpr uint64_t kObstacleWaitNs = 50000;
// want_zero: wait for the word to be 0; otherwise wait until (word & mask) == 0
GCC_D void await_row(const KParams &p, uint32_t row, unsigned long long mask, bool want_zero) {
    if (row == kNoRow || (p.flags & GCC_F_RETRY_IMMEDIATE)) return;
    const uint64_t t0 = gtimer();
    const uint64_t lim = p.spin_limit_ns < kObstacleWaitNs ? p.spin_limit_ns : kObstacleWaitNs;
    while (true) {
        unsigned long long w = ld_cg(p.meta + row);
        if (want_zero ? w == 0ull : (w & mask) == 0ull) return;
        if (gtimer() - t0 > lim) return;
        __nanosleep(64);
    }
}

// ---------------------------------------------------------------------------
// Latches of the slow_* variants (runtime.cuh:91-109), bounded.
// ---------------------------------------------------------------------------
GCC_D bool latch_acquire(const KParams &p, uint32_t row) {
    // CAS spin as in latch_lock (include/runtime.cuh:91-96), bounded. (A
    // test-and-test-and-set spin on a plain load starved diverged holder
    // lanes of the same warp here; every CAS attempt keeps the spinning path
    // stalled on L2 long enough for the holder to run its release.)
    unsigned *l = p.latch + row;
    if (atomicCAS(l, 0u, 1u) == 0u) { fence_acq_rel(); return true; }
    uint64_t t0 = gtimer();
    while (true) {
        if (atomicCAS(l, 0u, 1u) == 0u) { fence_acq_rel(); return true; }
        if (expired(t0, p.spin_limit_ns) || error_raised(p.ctr)) {
            set_error(p.ctr, GCC_ETIMEOUT, W_LATCH);
            return false;
        }
    }
}
GCC_D void latch_release(const KParams &p, uint32_t row) {
    fence_acq_rel();
    atomicExch(p.latch + row, 0u);
}

// Warp-aggregated timestamp allocation among the group leaders that arrive
// together (one atomic per warp instead of one per transaction).
GCC_D unsigned long long alloc_ts(Counters *c) {
    cg::coalesced_group act = cg::coalesced_threads();
    unsigned long long base = 0;
    if (act.thread_rank() == 0) base = atomicAdd(&c->ts, (unsigned long long)act.size());
    base = act.shfl(base, 0);
    return base + act.thread_rank();
}

// Per-attempt leader-side timing accumulators.
struct Clocks {
    unsigned long long ts, wait, mng;
};

// ===========================================================================
// 2PL no-wait / wait-die (twopl.cuh:233-322; slow_twopl.cuh:238-331)
// ===========================================================================
enum LockResult : int { L_OK = 0, L_DIE = 1, L_WAIT = 2, L_ERR = 3 };

template <bool WD>
GCC_D int tpl_shared(const KParams &p, uint32_t row, uint32_t tx) {
    unsigned long long *m = p.meta + row;
    if (WD) {
        unsigned long long w = ld_cg(m);
        if (w & tpl::kExcl) return tpl::holder(w) < tx ? L_DIE : L_WAIT;
    }
    unsigned long long old = atom_add_acq(m, 1ull);
    if (!(old & tpl::kExcl)) return L_OK;
    atomicAdd(m, ~0ull);  // undo the speculative reader increment
    if (!WD) return L_DIE;
    return tpl::holder(old) < tx ? L_DIE : L_WAIT;
}
template <bool WD>
GCC_D int tpl_excl(const KParams &p, uint32_t row, uint32_t tx) {
    unsigned long long old = atom_cas_acq(p.meta + row, 0ull, tpl::excl_word(tx));
    if (old == 0ull) return L_OK;
    if (!WD) return L_DIE;
    if (!(old & tpl::kExcl)) return L_DIE;  // shared holders: requester dies
    return tpl::holder(old) < tx ? L_DIE : L_WAIT;
}
// Latch variants: plain read/modify/write of the same word under a latch.
template <bool WD>
GCC_D int slow_tpl_lock(const KParams &p, uint32_t row, uint32_t tx, bool shared) {
    if (!latch_acquire(p, row)) return L_ERR;
    volatile unsigned long long *m = p.meta + row;
    unsigned long long w = *m;
    int r;
    if (shared) {
        if (!(w & tpl::kExcl)) { *m = w + 1ull; r = L_OK; }
        else r = (!WD || tpl::holder(w) < tx) ? L_DIE : L_WAIT;
    } else {
        if (w == 0ull) { *m = tpl::excl_word(tx); r = L_OK; }
        else if (!WD || !(w & tpl::kExcl)) r = L_DIE;
        else r = tpl::holder(w) < tx ? L_DIE : L_WAIT;
    }
    latch_release(p, row);
    return r;
}
template <bool SLOW>
GCC_D bool tpl_unlock(const KParams &p, uint32_t row, bool shared) {
    if (!SLOW) {
        // release: this lane's reads / writes of the row come before
        if (shared) red_add_rel(p.meta + row, ~0ull);
        else red_and_rel(p.meta + row, tpl::kReaders);
        return true;
    }
    if (shared) {
        if (!latch_acquire(p, row)) return false;
        volatile unsigned long long *m = p.meta + row;
        *m = *m - 1ull;
        latch_release(p, row);
    } else {
        // the exclusive holder is the only writer of the word
        // (slow_twopl.cuh:333-338 stores without the latch)
        fence_acq_rel();
        atomicExch(p.meta + row, 0ull);
    }
    return true;
}

template <bool WD, bool SLOW>
GCC_D int tpl_lock(const KParams &p, uint32_t row, uint32_t tx, bool rd) {
    return SLOW ? slow_tpl_lock<WD>(p, row, tx, rd)
                : (rd ? tpl_shared<WD>(p, row, tx) : tpl_excl<WD>(p, row, tx));
}

// First attempts take all locks at once (one ballot decides); after
// ordered_after failed attempts a retry takes them one request at a time,
// so that competing transactions cannot keep aborting each other. Both
// apply the scheme's rule: a conflict means abort (no-wait) or wait-or-die
// by transaction age (wait-die). Which locks a transaction takes and the
// rule applied to each never change; only the order of the acquisitions:
//   * by default a one-at-a-time retry takes every lock but one at once and
//     then the one whose request failed in the previous attempt: that lock
//     is contended, and taken last it is held the shortest time (taken in
//     request order, the reference's order, the hottest key of a Zipf
//     dataset comes first and is held while 15 more locks are taken one by
//     one, which made each writer of the hottest row cost ~15 us);
//   * GCC_F_REQUEST_ORDER and the latch variants keep request (= ascending
//     key) order (a latch variant's retries taking 15 latches at once kept
//     a starving transaction of a small hot table from ever committing);
//   * a lock plan (p.plan, set by the scheduler from its key-frequency
//     table) lists the hot requests: the others are taken at once, then the
//     hot ones one at a time, the hottest last.
template <int G, bool WD, bool SLOW, class TX>
GCC_D int attempt_tpl(const KParams &p, const Group<G> &g, const TX &s, uint32_t tx,
                      uint64_t pos, unsigned long long &dg, Clocks &ck, bool ordered) {
    constexpr int K = TX::K;
    uint32_t held = 0;
    bool fail = false, err = false;
    uint32_t obst = kNoRow;         // row whose lock request failed
    bool obst_x = false;            // ... and whether it was an exclusive request
    uint32_t obst_i = 0xFFFFFFFFu;  // ... and its request index
    uint64_t t0 = gtimer();
    long long cw = clock64();
    bool first = true;
    // planned: this attempt locks the requests outside the plan at once, then
    // the plan's requests in plan order; late bit k: op glane + k * G is planned
    bool planned = false;
    unsigned long long pl = 0;
    uint32_t late = 0;
    if constexpr (TX::MAXOPS == kMaxOps) {
        if (ordered && p.plan != nullptr) {
            planned = true;
            pl = __ldg(p.plan + tx);
        } else if (!SLOW && ordered && !(p.flags & GCC_F_REQUEST_ORDER) && s.obst_op) {
            // a one-entry plan: the request that failed last time, last
            planned = true;
            const unsigned long long i = s.obst_op - 1u;
            pl = (1ull << i) | (1ull << 16) | (i << 20);
        }
        if (planned) {
#pragma unroll
            for (int k = 0; k < K; ++k)
                if ((plan_mask(pl) >> (g.glane + k * G)) & 1u) late |= 1u << k;
        }
    }
    uint32_t pending = s.valid & ~late;
    // every pending request at once; a conflict fails the attempt (no-wait)
    // or, under wait-die, a younger holder makes the request wait
    auto lock_at_once = [&]() {
        while (true) {
#pragma unroll
            for (int k = 0; k < K; ++k) {
                if (!((pending >> k) & 1u) || fail || err) continue;
                int r = tpl_lock<WD, SLOW>(p, s.row[k], tx, (s.isread >> k) & 1u);
                if (r == L_OK) { held |= 1u << k; pending &= ~(1u << k); }
                else if (r == L_DIE) {
                    fail = true;
                    obst = s.row[k];
                    obst_x = !((s.isread >> k) & 1u);
                    obst_i = (uint32_t)(g.glane + k * G);
                }
                else if (r == L_ERR) err = true;
            }
            bool gf = g.any(fail), ge = g.any(err), gp = g.any(pending != 0u);
            if (ge) { fail = true; err = true; break; }
            if (gf || !gp) { fail = gf; break; }
            if (first) { first = false; cw = clock64(); }
            wait_pause();
            if (g.any(expired(t0, p.spin_limit_ns) || error_raised(p.ctr))) {
                if (g.glane == 0) set_error(p.ctr, GCC_ETIMEOUT, W_TPL_WD);
                fail = true; err = true; break;
            }
        }
    };
    if (ordered) {
        if (planned) lock_at_once();  // the requests outside the plan
        const uint32_t n_seq = planned ? plan_count(pl) : s.n;
        for (uint32_t j = 0; j < n_seq && !fail; ++j) {
            const uint32_t i = planned ? plan_op(pl, j) : j;
            const int owner = (int)(i % G), kk = (int)(i / G);
            int r = L_OK;
            if (g.glane == owner) {
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    if (k != kk || !((s.valid >> k) & 1u) || ((held >> k) & 1u)) continue;
                    while (true) {
                        r = tpl_lock<WD, SLOW>(p, s.row[k], tx, (s.isread >> k) & 1u);
                        if (r != L_WAIT) break;
                        if (first) { first = false; cw = clock64(); }
                        wait_pause();
                        if (expired(t0, p.spin_limit_ns) || error_raised(p.ctr)) {
                            set_error(p.ctr, GCC_ETIMEOUT, W_TPL_WD);
                            r = L_ERR;
                            break;
                        }
                    }
                    if (r == L_OK) held |= 1u << k;
                    else if (r == L_DIE) {
                        obst = s.row[k];
                        obst_x = !((s.isread >> k) & 1u);
                        obst_i = i;
                    }
                }
            }
            r = g.bcast(r, owner);
            if (r == L_DIE) fail = true;
            else if (r == L_ERR) { fail = true; err = true; }
        }
        // a plan only orders: whatever it did not list is locked now
        if (planned && !fail) {
            pending = s.valid & ~held;
            lock_at_once();
        }
    } else {
        lock_at_once();
    }
    if (!first) ck.wait += clock64() - cw;
    if (fail) {
#pragma unroll
        for (int k = 0; k < K; ++k)
            if ((held >> k) & 1u) tpl_unlock<SLOW>(p, s.row[k], (s.isread >> k) & 1u);
        if (err) return kGiveUp;
        if (!SLOW && !(p.flags & GCC_F_REQUEST_ORDER)) {
            const uint32_t fi = __reduce_min_sync(g.mask, obst_i);
            s.obst_op = fi == 0xFFFFFFFFu ? 0u : fi + 1u;
        }
        // an exclusive request waits for a free word, a shared one for the
        // exclusive holder to leave
        await_row(p, obst, tpl::kExcl, obst_x);
        return kAbort;
    }
    // (the fast variants' lock RMWs are acquire operations)
    if (SLOW) fence_acq_rel();
    // Serialization point: every lock is held. The leader's sequence number
    // is ordered after every lane's acquisition and before every lane's
    // release by the two warp syncs (lanes' memory operations are otherwise
    // unordered with respect to each other).
    if (p.flags & GCC_F_COMMIT_LOG) {
        g.sync();
        if (g.glane == 0) {
            p.commit_hi[tx] = atomicAdd(&p.ctr->seq, 1ull);
            p.commit_lo[tx] = 0ull;
        }
        g.sync();
    }
#pragma unroll
    for (int k = 0; k < K; ++k) {
        if (((s.valid & s.isread) >> k) & 1u) {
            read_image(p, row_ptr(p, s.row[k]), tx, pos, (uint32_t)(g.glane + k * G), dg);
        }
    }
    if (p.write_mode == GCC_WRITE_ROWCOPY) g.sync();
#pragma unroll
    for (int k = 0; k < K; ++k)
        if (((s.valid & ~s.isread) >> k) & 1u)
            apply_write<TX::kExt>(p, s.row[k], tx, pos, (uint32_t)(g.glane + k * G), s.readmask, dg);
    // (the fast variants' unlocks are release operations)
    if (SLOW) fence_acq_rel();
    bool uerr = false;
#pragma unroll
    for (int k = 0; k < K; ++k)
        if ((s.valid >> k) & 1u) uerr |= !tpl_unlock<SLOW>(p, s.row[k], (s.isread >> k) & 1u);
    return g.any(uerr) ? kGiveUp : kCommit;
}

// ===========================================================================
// Timestamp ordering (to.cuh:104-270; slow_to.cuh:137-238)
// ===========================================================================
enum OpResult : int { O_DONE = 0, O_FAIL = 1, O_RETRY = 2, O_ERR = 3 };

template <bool SLOW>
GCC_D int to_read(const KParams &p, uint32_t row, uint64_t ts, uint32_t tx, uint64_t pos,
                  uint32_t i, unsigned long long &dt) {
    unsigned long long *m = p.meta + row;
    if (SLOW) {
        if (!latch_acquire(p, row)) return O_ERR;
        unsigned long long x = *(volatile unsigned long long *)m;
        int r;
        if (tso::wts(x) > ts) r = O_FAIL;
        else if (x & tso::kUnc) r = O_RETRY;
        else {
            read_image(p, row_ptr(p, row), tx, pos, i, dt);
            uint64_t rts = tso::rts(x) > ts ? tso::rts(x) : ts;
            *(volatile unsigned long long *)m = tso::make(false, rts, tso::wts(x));
            r = O_DONE;
        }
        latch_release(p, row);
        return r;
    }
    unsigned long long x = ld_cg(m);
    if (tso::wts(x) > ts) return O_FAIL;
    if (x & tso::kUnc) return O_RETRY;  // wait for the older writer
    read_image(p, row_ptr(p, row), tx, pos, i, dt);
    if (tso::rts(x) >= ts) {
        // rts already covers this reader: only check the snapshot held
        fence_acq_rel();
        return ld_cg(m) == x ? O_DONE : O_RETRY;
    }
    unsigned long long nx = tso::make(false, ts, tso::wts(x));
    return atomicCAS(m, x, nx) == x ? O_DONE : O_RETRY;
}
template <bool SLOW>
GCC_D int to_write(const KParams &p, uint32_t row, uint64_t ts, unsigned long long &prev) {
    unsigned long long *m = p.meta + row;
    if (SLOW) {
        if (!latch_acquire(p, row)) return O_ERR;
        unsigned long long x = *(volatile unsigned long long *)m;
        int r;
        if (tso::rts(x) > ts || tso::wts(x) > ts || (x & tso::kUnc)) r = O_FAIL;
        else { prev = x; *(volatile unsigned long long *)m = tso::make(true, ts, ts); r = O_DONE; }
        latch_release(p, row);
        return r;
    }
    unsigned long long x = ld_cg(m);
    if (tso::rts(x) > ts || tso::wts(x) > ts || (x & tso::kUnc)) return O_FAIL;
    if (atomicCAS(m, x, tso::make(true, ts, ts)) != x) return O_RETRY;
    prev = x;
    return O_DONE;
}

template <int G, bool SLOW, class TX>
GCC_D int attempt_to(const KParams &p, const Group<G> &g, const TX &s, uint32_t tx,
                     uint64_t pos, unsigned long long &dg, Clocks &ck, bool ordered) {
    constexpr int K = TX::K;
    unsigned long long ts = 0;
    if (g.glane == 0) {
        long long c0 = clock64();
        ts = alloc_ts(p.ctr);
        ck.ts += clock64() - c0;
    }
    ts = g.bcast(ts, 0);
    if (ts > tso::kTsMax) {
        if (g.glane == 0) set_error(p.ctr, GCC_EOVERFLOW, 0);
        return kGiveUp;
    }
    uint32_t wrote = 0;
    unsigned long long prev[K];
    bool fail = false, err = false;
    uint64_t t0 = gtimer();
    bool first = true;
    long long cw = 0;
    uint32_t fail_i = 0xFFFFFFFFu;  // request index of this lane's failed op
    // A one-at-a-time retry visits every request but one at once first and
    // then the one that failed in the previous attempt, so a contended row
    // is held uncommitted the shortest time. Request order (the reference's)
    // instead under GCC_F_REQUEST_ORDER, in the latch variant, and for a
    // starving transaction: TO's conflicts are timestamp checks, and a
    // starving transaction that reached its contended row last kept meeting
    // younger readers there (one did not commit within the wait bound at
    // theta 0.8). late bit k: op glane + k * G is that one.
    uint32_t late = 0, late_i = 0xFFFFFFFFu;
    if constexpr (TX::MAXOPS == kMaxOps) {
        if (!SLOW && ordered && !(p.flags & GCC_F_REQUEST_ORDER) && s.obst_op) {
            late_i = s.obst_op - 1u;
#pragma unroll
            for (int k = 0; k < K; ++k)
                if ((uint32_t)(g.glane + k * G) == late_i) late |= 1u << k;
        }
    }
    uint32_t pending = s.valid & ~late;
    // One request: read (waits while an older writer's version is
    // uncommitted) or write (marks the row uncommitted with this ts).
    auto op = [&](int k) -> int {
        const uint32_t i = g.glane + k * G;
        int r;
        if ((s.isread >> k) & 1u) {
            unsigned long long dt = 0;
            r = to_read<SLOW>(p, s.row[k], ts, tx, pos, i, dt);
            if (r == O_DONE) dg += dt;
        } else {
            r = to_write<SLOW>(p, s.row[k], ts, prev[k]);
            if (r == O_DONE) wrote |= 1u << k;
        }
        if (r == O_FAIL) fail_i = i;
        return r;
    };
    // every pending request at once (reads of rows an older writer holds
    // uncommitted wait and retry)
    auto all_at_once = [&]() {
        while (true) {
#pragma unroll
            for (int k = 0; k < K; ++k) {
                if (!((pending >> k) & 1u) || fail || err) continue;
                int r = op(k);
                if (r == O_DONE) pending &= ~(1u << k);
                else if (r == O_FAIL) fail = true;
                else if (r == O_ERR) err = true;
            }
            bool ge = g.any(err), gf = g.any(fail), gp = g.any(pending != 0u);
            if (ge) { fail = err = true; break; }
            if (gf || !gp) { fail = gf; break; }
            if (first) { first = false; cw = clock64(); }
            wait_pause();
            if (g.any(expired(t0, p.spin_limit_ns) || error_raised(p.ctr))) {
                if (g.glane == 0) set_error(p.ctr, GCC_ETIMEOUT, W_TO_READ);
                fail = err = true; break;
            }
        }
    };
    if (ordered) {
        // Retries visit the requests one at a time, so two writers cannot
        // keep holding each other's rows uncommitted and aborting each other.
        const bool split = late_i != 0xFFFFFFFFu;
        if (split) all_at_once();  // the others
        const uint32_t n_seq = split ? 1u : s.n;
        for (uint32_t j = 0; j < n_seq && !fail; ++j) {
            const uint32_t i = split ? late_i : j;
            const int owner = (int)(i % G), kk = (int)(i / G);
            int r = O_DONE;
            if (g.glane == owner) {
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    if (k != kk || !((s.valid >> k) & 1u)) continue;
                    while (true) {
                        r = op(k);
                        if (r != O_RETRY) break;
                        if (first) { first = false; cw = clock64(); }
                        wait_pause();
                        if (expired(t0, p.spin_limit_ns) || error_raised(p.ctr)) {
                            set_error(p.ctr, GCC_ETIMEOUT, W_TO_READ);
                            r = O_ERR;
                            break;
                        }
                    }
                }
            }
            r = g.bcast(r, owner);
            if (r == O_FAIL) fail = true;
            else if (r == O_ERR) fail = err = true;
        }
    } else {
        all_at_once();
    }
    if (!SLOW && fail && !err && !(p.flags & GCC_F_REQUEST_ORDER)) {
        const uint32_t fi = __reduce_min_sync(g.mask, fail_i);
        s.obst_op = fi == 0xFFFFFFFFu ? 0u : fi + 1u;
    }
    if (!first) ck.wait += clock64() - cw;
    if (fail) {
        // restore the words this attempt marked uncommitted (to.cuh:255-270)
#pragma unroll
        for (int k = 0; k < K; ++k)
            if ((wrote >> k) & 1u) atomicExch(p.meta + s.row[k], prev[k]);
        fence_acq_rel();
        return err ? kGiveUp : kAbort;
    }
    // Serialization key: (batch, timestamp); timestamps restart per batch.
    if ((p.flags & GCC_F_COMMIT_LOG) && g.glane == 0) {
        p.commit_hi[tx] = p.batch_st;
        p.commit_lo[tx] = ts;
    }
    if (p.write_mode == GCC_WRITE_ROWCOPY) g.sync();
#pragma unroll
    for (int k = 0; k < K; ++k)
        if ((wrote >> k) & 1u) apply_write<TX::kExt>(p, s.row[k], tx, pos, g.glane + k * G, s.readmask, dg);
    fence_acq_rel();
#pragma unroll
    for (int k = 0; k < K; ++k)
        if ((wrote >> k) & 1u) atomicExch(p.meta + s.row[k], tso::make(false, ts, ts));
    return kCommit;
}

// ===========================================================================
// MVCC (mvcc.cuh:113-297). Requests run one at a time in program order (the
// reader waits on any uncommitted version, as in the reference, and
// ascending-key access keeps those waits acyclic). Two reference defects are
// not reproduced: the base row is updated at commit (mvcc.cuh:143 leaves the
// copy commented out) and each version owns a full row image (mvcc.cuh:142
// strides the version data by sizeof(version_node)).
// ===========================================================================
template <bool SLOW>
GCC_D int mvcc_read(const KParams &p, uint32_t row, uint64_t ts, uint32_t tx, uint64_t pos,
                    uint32_t i, unsigned long long &dt) {
    unsigned long long *m = p.meta + row;
    if (SLOW && !latch_acquire(p, row)) return O_ERR;
    unsigned long long x = SLOW ? *(volatile unsigned long long *)m : ld_cg(m);
    int r;
    if (x & tso::kUnc) {
        r = O_RETRY;
    } else if (tso::wts(x) <= ts) {
        read_image(p, row_ptr(p, row), tx, pos, i, dt);
        if (tso::rts(x) >= ts) {
            fence_acq_rel();
            r = (SLOW || ld_cg(m) == x) ? O_DONE : O_RETRY;
        } else if (SLOW) {
            *(volatile unsigned long long *)m = tso::make(false, ts, tso::wts(x));
            r = O_DONE;
        } else {
            r = atomicCAS(m, x, tso::make(false, ts, tso::wts(x))) == x ? O_DONE : O_RETRY;
        }
    } else {
        // walk the version chain to the newest version with wts <= ts
        unsigned node = ld_cg(p.turn + row);
        unsigned hops = 0;
        while (node != kNoRow && tso::wts(ld_cg(p.ver_ts + node)) > ts && hops < 0x1000000u) {
            node = ld_cg(p.ver_prev + node);
            ++hops;
        }
        if (node == kNoRow || hops >= 0x1000000u) {
            set_error(p.ctr, GCC_EFORMAT, W_MVCC_READ);  // broken chain
            r = O_ERR;
        } else {
            read_image(p, p.ver_data + (size_t)node * p.wslot, tx, pos, i, dt);
            fence_acq_rel();
            r = (SLOW || ld_cg(m) == x) ? O_DONE : O_RETRY;
        }
    }
    if (SLOW) latch_release(p, row);
    return r;
}

template <int G, bool SLOW, class TX>
GCC_D int attempt_mvcc(const KParams &p, const Group<G> &g, const TX &s, uint32_t tx,
                       uint64_t pos, unsigned long long &dg, Clocks &ck, bool ordered) {
    constexpr int K = TX::K;
    unsigned long long ts = 0;
    if (g.glane == 0) {
        long long c0 = clock64();
        ts = alloc_ts(p.ctr);
        ck.ts += clock64() - c0;
    }
    ts = g.bcast(ts, 0);
    if (ts > tso::kTsMax) {
        if (g.glane == 0) set_error(p.ctr, GCC_EOVERFLOW, 0);
        return kGiveUp;
    }
    uint32_t wrote = 0;
    unsigned long long prev[K];
    bool fail = false, err = false;
    for (uint32_t i = 0; i < s.n; ++i) {
        const int owner = (int)(i % G);
        const int kk = (int)(i / G);
        if (g.glane == owner) {
            uint64_t t0 = gtimer();
            long long cw = clock64();
#pragma unroll
            for (int k = 0; k < K; ++k) {
                if (k != kk) continue;
                while (true) {
                    int r;
                    if ((s.isread >> k) & 1u) {
                        unsigned long long dt = 0;
                        r = mvcc_read<SLOW>(p, s.row[k], ts, tx, pos, i, dt);
                        if (r == O_DONE) dg += dt;
                    } else {
                        r = to_write<SLOW>(p, s.row[k], ts, prev[k]);
                        if (r == O_DONE) wrote |= 1u << k;
                    }
                    if (r == O_DONE) break;
                    if (r == O_FAIL) { fail = true; break; }
                    if (r == O_ERR) { err = true; break; }
                    wait_pause();
                    if (expired(t0, p.spin_limit_ns) || error_raised(p.ctr)) {
                        set_error(p.ctr, GCC_ETIMEOUT, W_MVCC_READ);
                        err = true;
                        break;
                    }
                }
            }
            ck.wait += clock64() - cw;
        }
        bool gf = g.any(fail), ge = g.any(err);
        if (gf || ge) { fail = true; err = ge; break; }
    }
    if (fail) {
#pragma unroll
        for (int k = 0; k < K; ++k)
            if ((wrote >> k) & 1u) atomicExch(p.meta + s.row[k], prev[k]);
        fence_acq_rel();
        return err ? kGiveUp : kAbort;
    }
    // Serialization key: (batch, timestamp); timestamps restart per batch.
    if ((p.flags & GCC_F_COMMIT_LOG) && g.glane == 0) {
        p.commit_hi[tx] = p.batch_st;
        p.commit_lo[tx] = ts;
    }
    if (p.write_mode == GCC_WRITE_ROWCOPY) g.sync();
#pragma unroll
    for (int k = 0; k < K; ++k) {
        if (!((wrote >> k) & 1u)) continue;
        uint32_t i = g.glane + k * G;
        uint32_t row = s.row[k];
        // push the current base row as the version it replaces, link it,
        // then install the new base row and publish (uncommitted -> 0)
        uint32_t node = (uint32_t)(pos * p.slot_ops + i);
        copy_image(p, p.ver_data + (size_t)node * p.wslot, row_ptr(p, row));
        p.ver_ts[node] = prev[k];
        p.ver_prev[node] = ld_cg(p.turn + row);
        fence_acq_rel();
        atomicExch(p.turn + row, node);
        apply_write<TX::kExt>(p, row, tx, pos, i, s.readmask, dg);
        fence_acq_rel();
        atomicExch(p.meta + row, tso::make(false, ts, ts));
    }
    return kCommit;
}

// ===========================================================================
// Silo (silo.cuh:116-338; slow_silo.cuh:188-326). The commit timestamp is
// max(read-set ts, current write-set ts) + 1 as in Silo; the reference takes
// the write-set term from a field Write never sets (silo.cuh:306-310), which
// lets a record's ts repeat and a stale read validate.
// ===========================================================================
template <bool SLOW>
GCC_D int silo_read(const KParams &p, uint32_t row, uint32_t tx, uint64_t pos, uint32_t i,
                    unsigned long long &dt, unsigned long long &ts) {
    unsigned long long *m = p.meta + row;
    if (SLOW) {
        if (!latch_acquire(p, row)) return O_ERR;
        unsigned long long x = *(volatile unsigned long long *)m;
        int r = O_RETRY;
        if (!(x & silo::kLock)) { read_image(p, row_ptr(p, row), tx, pos, i, dt); ts = silo::ts(x); r = O_DONE; }
        latch_release(p, row);
        return r;
    }
    unsigned long long x1 = ld_cg(m);
    if (x1 & silo::kLock) return O_RETRY;
    fence_acq_rel();
    read_image(p, row_ptr(p, row), tx, pos, i, dt);
    fence_acq_rel();
    unsigned long long x2 = ld_cg(m);
    if (x1 != x2) return O_RETRY;
    ts = silo::ts(x1);
    return O_DONE;
}
// No-wait write lock: O_DONE (cur = word before locking), O_FAIL if locked.
template <bool SLOW>
GCC_D int occ_lock(const KParams &p, uint32_t row, unsigned long long lockbit,
                   unsigned long long &cur) {
    unsigned long long *m = p.meta + row;
    if (SLOW) {
        if (!latch_acquire(p, row)) return O_ERR;
        unsigned long long x = *(volatile unsigned long long *)m;
        int r = O_FAIL;
        if (!(x & lockbit)) { *(volatile unsigned long long *)m = x | lockbit; cur = x; r = O_DONE; }
        latch_release(p, row);
        return r;
    }
    for (int tries = 0; tries < 1 << 20; ++tries) {
        unsigned long long x = ld_cg(m);
        if (x & lockbit) return O_FAIL;
        if (atomicCAS(m, x, x | lockbit) == x) { cur = x; return O_DONE; }
    }
    set_error(p.ctr, GCC_ETIMEOUT, W_CAS);
    return O_ERR;
}

// Lock the write set, no-wait (silo.cuh:268-281, tictoc.cuh:269-282). First
// attempts lock in parallel; retries lock one request at a time in request
// order. `cts` accumulates f(word before locking) over the locked words.
template <int G, bool SLOW, bool TICTOC, class TX>
GCC_D void occ_lock_writes(const KParams &p, const Group<G> &g, const TX &s,
                           uint32_t writes, bool ordered, uint32_t &held,
                           unsigned long long &cts, bool &fail, bool &err, uint32_t &obst) {
    constexpr int K = TX::K;
    const unsigned long long lockbit = TICTOC ? tictoc::kLock : silo::kLock;
    if (!ordered) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            if (!((writes >> k) & 1u) || fail || err) continue;
            unsigned long long cur;
            int r = occ_lock<SLOW>(p, s.row[k], lockbit, cur);
            if (r == O_DONE) {
                held |= 1u << k;
                unsigned long long c = TICTOC ? tictoc::rts(cur) + 1ull : silo::ts(cur);
                cts = cts > c ? cts : c;
            } else if (r == O_FAIL) { fail = true; obst = s.row[k]; }
            else err = true;
        }
        return;
    }
    for (uint32_t i = 0; i < s.n; ++i) {
        const int owner = (int)(i % G), kk = (int)(i / G);
        int r = O_DONE;
        if (g.glane == owner) {
#pragma unroll
            for (int k = 0; k < K; ++k) {
                if (k != kk || !((writes >> k) & 1u)) continue;
                unsigned long long cur;
                r = occ_lock<SLOW>(p, s.row[k], lockbit, cur);
                if (r == O_DONE) {
                    held |= 1u << k;
                    unsigned long long c = TICTOC ? tictoc::rts(cur) + 1ull : silo::ts(cur);
                    cts = cts > c ? cts : c;
                } else if (r == O_FAIL) obst = s.row[k];
            }
        }
        r = g.bcast(r, owner);
        if (r == O_FAIL) { fail = true; break; }
        if (r == O_ERR) { err = true; break; }
    }
}

template <int G, bool SLOW, class TX>
GCC_D int attempt_silo(const KParams &p, const Group<G> &g, const TX &s, uint32_t tx,
                       uint64_t pos, unsigned long long &dg, Clocks &ck, bool ordered) {
    constexpr int K = TX::K;
    unsigned long long rec[K];
    uint32_t reads = s.valid & s.isread, writes = s.valid & ~s.isread;
    uint32_t pending = reads, held = 0;
    bool fail = false, err = false;
    // read phase: consistent snapshots (silo.cuh:223-259)
    uint64_t t0 = gtimer();
    bool first = true;
    long long cw = 0;
    while (true) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            if (!((pending >> k) & 1u) || err) continue;
            unsigned long long dt = 0;
            int r = silo_read<SLOW>(p, s.row[k], tx, pos, g.glane + k * G, dt, rec[k]);
            if (r == O_DONE) { pending &= ~(1u << k); dg += dt; }
            else if (r == O_ERR) err = true;
        }
        bool ge = g.any(err), gp = g.any(pending != 0u);
        if (ge) return kGiveUp;
        if (!gp) break;
        if (first) { first = false; cw = clock64(); }
        wait_pause();
        if (g.any(expired(t0, p.spin_limit_ns) || error_raised(p.ctr))) {
            if (g.glane == 0) set_error(p.ctr, GCC_ETIMEOUT, W_SILO_READ);
            return kGiveUp;
        }
    }
    if (!first) ck.wait += clock64() - cw;
    // validation: lock the write set, no-wait (silo.cuh:268-281)
    unsigned long long cts = 0;
    uint32_t obst = kNoRow;
    occ_lock_writes<G, SLOW, false>(p, g, s, writes, ordered, held, cts, fail, err, obst);
    bool gf = g.any(fail), ge = g.any(err);
    if (!gf && !ge) {
        fence_acq_rel();
        // Serialization point: write set locked (by every lane), read set not
        // yet validated (by any lane); the warp syncs order the leader's
        // sequence number between the two.
        if (p.flags & GCC_F_COMMIT_LOG) {
            g.sync();
            if (g.glane == 0) {
                p.commit_hi[tx] = atomicAdd(&p.ctr->seq, 1ull);
                p.commit_lo[tx] = 0ull;
            }
            g.sync();
        }
#pragma unroll
        for (int k = 0; k < K; ++k) {
            if (!((reads >> k) & 1u)) continue;
            unsigned long long x = ld_cg(p.meta + s.row[k]);
            if (silo::ts(x) != rec[k] || (x & silo::kLock)) {
                fail = true;
                if (x & silo::kLock) obst = s.row[k];
            }
            cts = cts > rec[k] ? cts : rec[k];
        }
        gf = g.any(fail);
    }
    if (gf || ge) {
#pragma unroll
        for (int k = 0; k < K; ++k)
            if ((held >> k) & 1u) atomicAnd(p.meta + s.row[k], ~silo::kLock);
        fence_acq_rel();
        return ge ? kGiveUp : kAbort;
    }
    cts = g.maxv(cts) + 1ull;
    if (p.write_mode == GCC_WRITE_ROWCOPY) g.sync();
#pragma unroll
    for (int k = 0; k < K; ++k)
        if ((writes >> k) & 1u) apply_write<TX::kExt>(p, s.row[k], tx, pos, g.glane + k * G, s.readmask, dg);
    fence_acq_rel();
#pragma unroll
    for (int k = 0; k < K; ++k)
        if ((writes >> k) & 1u) atomicExch(p.meta + s.row[k], cts);
    return kCommit;
}

// ===========================================================================
// TicToc (tictoc.cuh:115-368; slow_tictoc.cuh)
// ===========================================================================
template <bool SLOW>
GCC_D int tictoc_read(const KParams &p, uint32_t row, uint32_t tx, uint64_t pos, uint32_t i,
                      unsigned long long &dt, unsigned long long &wts, unsigned long long &rts) {
    unsigned long long *m = p.meta + row;
    if (SLOW) {
        if (!latch_acquire(p, row)) return O_ERR;
        unsigned long long x = *(volatile unsigned long long *)m;
        int r = O_RETRY;
        if (!(x & tictoc::kLock)) {
            read_image(p, row_ptr(p, row), tx, pos, i, dt);
            wts = tictoc::wts(x); rts = tictoc::rts(x); r = O_DONE;
        }
        latch_release(p, row);
        return r;
    }
    unsigned long long x1 = ld_cg(m);
    if (x1 & tictoc::kLock) return O_RETRY;
    fence_acq_rel();
    read_image(p, row_ptr(p, row), tx, pos, i, dt);
    fence_acq_rel();
    if (ld_cg(m) != x1) return O_RETRY;
    wts = tictoc::wts(x1);
    rts = tictoc::rts(x1);
    return O_DONE;
}
// Extend a read version's rts to cover commit_ts (tictoc.cuh:302-340).
template <bool SLOW>
GCC_D int tictoc_extend(const KParams &p, uint32_t row, unsigned long long rwts,
                        unsigned long long cts) {
    unsigned long long *m = p.meta + row;
    for (int tries = 0; tries < 1 << 20; ++tries) {
        if (SLOW && !latch_acquire(p, row)) return O_ERR;
        unsigned long long x = SLOW ? *(volatile unsigned long long *)m : ld_cg(m);
        unsigned long long wts = tictoc::wts(x), rts = tictoc::rts(x);
        int r;
        if (wts != rwts || (rts <= cts && (x & tictoc::kLock))) {
            r = O_FAIL;
        } else if (rts > cts) {
            r = O_DONE;
        } else {
            unsigned long long delta = cts - wts;
            unsigned long long shift = delta - (delta & 0x7FFFull);
            unsigned long long nx = tictoc::make(false, delta - shift, wts + shift);
            if (SLOW) { *(volatile unsigned long long *)m = nx; r = O_DONE; }
            else r = atomicCAS(m, x, nx) == x ? O_DONE : O_RETRY;
        }
        if (SLOW) latch_release(p, row);
        if (r != O_RETRY) return r;
    }
    set_error(p.ctr, GCC_ETIMEOUT, W_TICTOC_EXT);
    return O_ERR;
}

template <int G, bool SLOW, class TX>
GCC_D int attempt_tictoc(const KParams &p, const Group<G> &g, const TX &s, uint32_t tx,
                         uint64_t pos, unsigned long long &dg, Clocks &ck, bool ordered) {
    constexpr int K = TX::K;
    unsigned long long rw[K], rr[K];
    uint32_t reads = s.valid & s.isread, writes = s.valid & ~s.isread;
    uint32_t pending = reads, held = 0;
    bool fail = false, err = false;
    uint64_t t0 = gtimer();
    bool first = true;
    long long cw = 0;
    while (true) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            if (!((pending >> k) & 1u) || err) continue;
            unsigned long long dt = 0;
            int r = tictoc_read<SLOW>(p, s.row[k], tx, pos, g.glane + k * G, dt, rw[k], rr[k]);
            if (r == O_DONE) { pending &= ~(1u << k); dg += dt; }
            else if (r == O_ERR) err = true;
        }
        bool ge = g.any(err), gp = g.any(pending != 0u);
        if (ge) return kGiveUp;
        if (!gp) break;
        if (first) { first = false; cw = clock64(); }
        wait_pause();
        if (g.any(expired(t0, p.spin_limit_ns) || error_raised(p.ctr))) {
            if (g.glane == 0) set_error(p.ctr, GCC_ETIMEOUT, W_TICTOC_READ);
            return kGiveUp;
        }
    }
    if (!first) ck.wait += clock64() - cw;
    unsigned long long cts = 0;
    uint32_t obst = kNoRow;
    occ_lock_writes<G, SLOW, true>(p, g, s, writes, ordered, held, cts, fail, err, obst);
    bool gf = g.any(fail), ge = g.any(err);
    if (!gf && !ge) {
#pragma unroll
        for (int k = 0; k < K; ++k)
            if ((reads >> k) & 1u) cts = cts > rw[k] ? cts : rw[k];
        cts = g.maxv(cts);
#pragma unroll
        for (int k = 0; k < K; ++k) {
            if (!((reads >> k) & 1u) || fail || err) continue;
            if (rr[k] >= cts) continue;
            int r = tictoc_extend<SLOW>(p, s.row[k], rw[k], cts);
            if (r == O_FAIL) { fail = true; obst = s.row[k]; }
            else if (r == O_ERR) err = true;
        }
        gf = g.any(fail);
        ge = g.any(err);
    }
    if (gf || ge) {
#pragma unroll
        for (int k = 0; k < K; ++k)
            if ((held >> k) & 1u) atomicAnd(p.meta + s.row[k], ~tictoc::kLock);
        fence_acq_rel();
        return ge ? kGiveUp : kAbort;
    }
    // Serialization key: (batch, commit_ts, order of validation among equal
    // commit_ts). Within a batch commit_ts <= commits + 1 < 2^32.
    if (p.flags & GCC_F_COMMIT_LOG) {
        g.sync();
        if (g.glane == 0) {
            p.commit_hi[tx] = p.batch_st;
            p.commit_lo[tx] = (cts << 32) | (atomicAdd(&p.ctr->seq, 1ull) & 0xFFFFFFFFull);
        }
        g.sync();
    }
    if (p.write_mode == GCC_WRITE_ROWCOPY) g.sync();
#pragma unroll
    for (int k = 0; k < K; ++k)
        if ((writes >> k) & 1u) apply_write<TX::kExt>(p, s.row[k], tx, pos, g.glane + k * G, s.readmask, dg);
    fence_acq_rel();
#pragma unroll
    for (int k = 0; k < K; ++k)
        if ((writes >> k) & 1u) atomicExch(p.meta + s.row[k], tictoc::make(false, 0, cts));
    return kCommit;
}

// ===========================================================================
// GaccO / GPUTx: deterministic execution in a precomputed order. Each access
// (row, position p in that row's ordered access list) waits until the row's
// turn equals p, performs the read or write, and passes the turn to p + 1
// (gacco.cuh:156-175; GPUTx's rank launches become the same hand-off over the
// (rank, tx) order, which also orders same-rank conflicts by tx index).
// ===========================================================================
template <int G, class TX>
GCC_D int attempt_ordered(const KParams &p, const Group<G> &g, const TX &s, uint32_t tx,
                          uint64_t pos, unsigned long long &dg, Clocks &ck, bool ordered) {
    constexpr int K = TX::K;
    uint32_t mypos[K];
#pragma unroll
    for (int k = 0; k < K; ++k)
        mypos[k] = ((s.valid >> k) & 1u) ? p.op_pos[pos * p.slot_ops + g.glane + k * G] : 0u;
    uint32_t pending = s.valid;
    unsigned long long done_ops = 0;
    const bool rowcopy = p.write_mode == GCC_WRITE_ROWCOPY;
    uint64_t t0 = gtimer();
    bool first = true;
    long long cw = 0;
    while (true) {
        unsigned long long mine = 0;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            if (!((pending >> k) & 1u)) continue;
            uint32_t i = g.glane + k * G;
            bool rd = (s.isread >> k) & 1u;
            if (!rd && rowcopy) {
                int src = rowcopy_src(s.readmask, i);
                if (src >= 0 && !((done_ops >> src) & 1ull)) continue;
            }
            // acquire: the predecessor's access to the row is visible
            if (ld_acquire(p.turn + s.row[k]) != mypos[k]) continue;
            if (rd) {
                read_image(p, row_ptr(p, s.row[k]), tx, pos, i, dg);
            } else {
                apply_write<TX::kExt>(p, s.row[k], tx, pos, i, s.readmask, dg);
            }
            // release: this access comes before the successor's
            st_release(p.turn + s.row[k], mypos[k] + 1u);
            pending &= ~(1u << k);
            mine |= 1ull << i;
        }
        done_ops |= g.orv(mine);
        if (rowcopy) g.sync();
        if (!g.any(pending != 0u)) break;
        if (first) { first = false; cw = clock64(); }
        wait_pause();
        if (g.any(expired(t0, p.spin_limit_ns) || error_raised(p.ctr))) {
            if (g.glane == 0) set_error(p.ctr, GCC_ETIMEOUT, W_TURN);
            return kGiveUp;
        }
    }
    if (!first) ck.wait += clock64() - cw;
    if ((p.flags & GCC_F_COMMIT_LOG) && g.glane == 0) {
        p.commit_hi[tx] = p.batch_st + pos;
        p.commit_lo[tx] = 0ull;
    }
    return kCommit;
}

template <int SCH, int G, class TX>
GCC_D int attempt(const KParams &p, const Group<G> &g, const TX &s, uint32_t tx,
                  uint64_t pos, unsigned long long &dg, Clocks &ck, bool ordered) {
    if constexpr (SCH == S_TPL_NW) return attempt_tpl<G, false, false>(p, g, s, tx, pos, dg, ck, ordered);
    else if constexpr (SCH == S_TPL_WD) return attempt_tpl<G, true, false>(p, g, s, tx, pos, dg, ck, ordered);
    else if constexpr (SCH == S_SLOW_TPL_NW) return attempt_tpl<G, false, true>(p, g, s, tx, pos, dg, ck, ordered);
    else if constexpr (SCH == S_SLOW_TPL_WD) return attempt_tpl<G, true, true>(p, g, s, tx, pos, dg, ck, ordered);
    else if constexpr (SCH == S_TO) return attempt_to<G, false>(p, g, s, tx, pos, dg, ck, ordered);
    else if constexpr (SCH == S_SLOW_TO) return attempt_to<G, true>(p, g, s, tx, pos, dg, ck, ordered);
    else if constexpr (SCH == S_MVCC) return attempt_mvcc<G, false>(p, g, s, tx, pos, dg, ck, ordered);
    else if constexpr (SCH == S_SLOW_MVCC) return attempt_mvcc<G, true>(p, g, s, tx, pos, dg, ck, ordered);
    else if constexpr (SCH == S_SILO) return attempt_silo<G, false>(p, g, s, tx, pos, dg, ck, ordered);
    else if constexpr (SCH == S_SLOW_SILO) return attempt_silo<G, true>(p, g, s, tx, pos, dg, ck, ordered);
    else if constexpr (SCH == S_TICTOC) return attempt_tictoc<G, false>(p, g, s, tx, pos, dg, ck, ordered);
    else if constexpr (SCH == S_SLOW_TICTOC) return attempt_tictoc<G, true>(p, g, s, tx, pos, dg, ck, ordered);
    else return attempt_ordered<G>(p, g, s, tx, pos, dg, ck, ordered);
}

__host__ __device__ constexpr bool is_ordered(int s) { return s == S_GACCO || s == S_GPUTX; }

// Attempts before retries switch to one request at a time (the caller can
// move the switch of 2PL / TO with gcc_run_params.ordered_after).
// Retries take their requests in parallel like the first attempt: Silo and
// TicToc always, TO and 2PL for their first 15 retries, after which they go
// one request at a time (starting from the request that failed last time,
// see attempt_tpl / attempt_to; in key order under GCC_F_REQUEST_ORDER, which
// is what the measurements below used). The starvation control bounds the
// cycles that made fully parallel retries livelock. Measured (10,485,760
// rows, r 0.9) against ordering from the first retry: silo / tictoc +40 %
// at theta 0.6 and +25-50 % at 0.8-0.99; TO 22.9 -> 57 M tx/s at 0.6 and
// unchanged at 0.8-0.99; tpl_nw 58 -> 67 M at 0.6, -5 % at 0.8, unchanged
// at 0.9-0.99 (never ordering 2PL / TO gives 98 M at 0.6 but -35 % at 0.8
// and above). The latch variants follow their fast counterparts (ordering
// them from the first retry made every retry 16 dependent latch round trips
// and left slow_tpl_nw at a tenth of tpl_nw at theta 0.6); MVCC and the
// ordered schemes keep requests in program order.
__host__ __device__ constexpr unsigned ordered_after(int s) {
    return (s == S_SILO || s == S_TICTOC || s == S_SLOW_SILO || s == S_SLOW_TICTOC)
               ? 0xFFFFFFFFu
               : ((s == S_TO || s == S_TPL_NW || s == S_TPL_WD || s == S_SLOW_TO ||
                   s == S_SLOW_TPL_NW || s == S_SLOW_TPL_WD)
                      ? 16u
                      : 1u);
}

// ===========================================================================
// The persistent transaction kernel.
// ===========================================================================
template <int SCH, int G, int MO = kMaxOps>
__global__ void __launch_bounds__(1024, 1) ycsb_kernel(const __grid_constant__ KParams p) {
    // Block-level histogram and metric sums (flushed once at exit) keep the
    // per-thread register budget for the transaction itself.
    __shared__ unsigned s_hist[kHistBuckets];
    __shared__ unsigned long long s_met[8];
    for (int i = threadIdx.x; i < kHistBuckets; i += blockDim.x) s_hist[i] = 0u;
    if (threadIdx.x < 8) s_met[threadIdx.x] = 0ull;
    __syncthreads();

    const Group<G> g;
    using TX = TxOps<G, MO>;
    constexpr int K = TX::K;

    // Positions come from 32 striped ticket counters (stripe j hands out
    // j, j + 32, j + 64, ... in increasing order, each counter on its own
    // 128-byte line): one same-address atomic per transaction on a single
    // counter was the main latency term at low contention. A group starts on
    // stripe (group id % 32) and moves to the next stripe when its stripe is
    // exhausted. Within a stripe positions are taken in order and a group
    // runs one position at a time, so the lowest unfinished position is
    // always held by a running group (the ordered schemes' hand-off stays
    // live).
    const unsigned gid = (blockIdx.x * blockDim.x + threadIdx.x) / G;
    unsigned stripe = gid % kTicketStripes, tried = 0;
    while (true) {
        unsigned long long pos = 0;
        unsigned stop = 0;
        if (g.glane == 0) {
            // admission pause: while some transaction is starving (it has
            // aborted starve_limit times), take no new transaction, so the
            // contention around it drains and it commits. The pause is
            // advisory: after spin_limit_ns admissions resume regardless.
            if (p.starve_limit && ld_volatile(&p.ctr->starving) != 0u) {
                const uint64_t tw = gtimer();
                while (ld_volatile(&p.ctr->starving) != 0u) {
                    if (error_raised(p.ctr) || expired(tw, p.spin_limit_ns)) break;
                    __nanosleep(1000);
                }
            }
            while (true) {
                unsigned long long t = atomicAdd(&p.ctr->tickets[stripe * 16], 1ull);
                pos = t * kTicketStripes + stripe;
                if (pos < p.batch_n) break;
                if (++tried >= kTicketStripes) { stop = 1u; break; }
                stripe = (stripe + 1) % kTicketStripes;
            }
            // device queue: wait (bounded) until the position is admitted
            if (!stop && p.queue_tail) {
                const uint64_t tq = gtimer();
                while (pos >= *p.queue_tail) {
                    if (error_raised(p.ctr) || expired(tq, p.spin_limit_ns)) {
                        set_error(p.ctr, GCC_ETIMEOUT, W_QUEUE);
                        stop = 1u;
                        break;
                    }
                    __nanosleep(256);
                }
            }
            if (error_raised(p.ctr)) stop = 1u;
        }
        stop = g.bcast(stop, 0);
        if (stop) break;
        pos = g.bcast(pos, 0);
        const uint32_t tx = p.order ? __ldg(p.order + p.batch_st + pos) : p.batch_st + (uint32_t)pos;
        const long long c_start = clock64();
        const uint64_t t_start = gtimer();

        // ---- requests and index probes --------------------------------
        TX s;
        unsigned long long n64;
        const gcc_ycsb_tx *T = nullptr;
        uint32_t beg = 0;
        if constexpr (MO == kMaxOps) {
            T = p.txs + tx;
            // With a device queue the records of later batches are still
            // being copied in while earlier ones run: read them through L2
            // (a line cached in L1 next to an earlier record could predate
            // the copy).
            n64 = p.queue_tail ? __ldcg((const unsigned long long *)&T->request_cnt)
                               : __ldg(&T->request_cnt);
        } else {
            beg = __ldg(p.tx_off + tx);
            n64 = (unsigned long long)(__ldg(p.tx_off + tx + 1) - beg);
        }
        if (n64 > (unsigned long long)MO) {
            if (g.glane == 0) set_error(p.ctr, GCC_EFORMAT, 0);
            break;
        }
        s.n = (uint32_t)n64;
        s.valid = s.isread = 0;
        s.obst_op = 0;
        bool miss = false;
        unsigned long long myreads = 0;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const uint32_t i = g.glane + k * G;
            s.row[k] = kNoRow;
            if (i < s.n) {
                int2 rq;
                if constexpr (MO == kMaxOps)
                    rq = p.queue_tail ? __ldcg((const int2 *)&T->requests[i])
                                      : __ldg((const int2 *)&T->requests[i]);
                else rq = __ldg((const int2 *)(p.reqs + beg + i));
                s.valid |= 1u << k;
                if (rq.x > 0) { s.isread |= 1u << k; myreads |= 1ull << i; }
                if constexpr (is_ordered(SCH)) {
                    s.row[k] = __ldg(p.op_row + pos * p.slot_ops + i);
                } else {
                    s.row[k] = index_find(p, (uint32_t)rq.y);
                }
                miss |= s.row[k] == kNoRow;
            }
        }
        s.readmask = g.orv(myreads);
        if (g.any(miss)) {
            if (g.glane == 0) set_error(p.ctr, GCC_EKEY, 0);
            break;
        }
        const long long c_after_idx = clock64();

        // ---- attempt / retry loop (benchmark/ycsb.cu:51-106) -------------
        unsigned attempts = 0;
        int st = kGiveUp;
        Clocks ck{0, 0, 0};
        unsigned long long dg = 0, c_abort = 0;
        long long c_attempt = c_after_idx;
        bool starving = false;
        // (the caller's ordered_from applies to the schemes that switch, 2PL / TO)
        const unsigned ord_from = (p.ordered_from && ordered_after(SCH) == 16u)
                                      ? p.ordered_from - 1u : ordered_after(SCH);
        while (true) {
            dg = 0;
            c_attempt = clock64();
            st = attempt<SCH, G>(p, g, s, tx, pos, dg, ck, attempts >= ord_from);
            if (st != kAbort) break;
            ++attempts;
            if (p.starve_limit && attempts == p.starve_limit) {
                starving = true;
                if (g.glane == 0) atomicAdd(&p.ctr->starving, 1u);
            }
            // a starving TO transaction retries in request order (see
            // attempt_to); starving 2PL ones keep the failed lock last, which
            // is what lets the hot rows' writers through
            if constexpr (SCH == S_TO) {
                if (starving) s.obst_op = 0;
            }
            // A transaction still aborting after 4 x starve_limit attempts
            // retries only while it holds the starvation token: the others
            // at that stage wait between attempts, holding nothing, so the
            // holder meets only the in-flight work below that stage, which
            // drains (admissions are paused) or reaches it in turn. One
            // holder at a time guarantees progress for transactions whose
            // retries would otherwise keep invalidating each other.
            if (starving && attempts >= 4u * p.starve_limit) {
                unsigned bad = 0;
                if (g.glane == 0) {
                    const unsigned me = tx + 1u;
                    const uint64_t tw = gtimer();
                    while (true) {
                        const unsigned h = atomicCAS(&p.ctr->starve_token, 0u, me);
                        if (h == 0u || h == me) break;
                        if (error_raised(p.ctr)) { bad = 1; break; }
                        if (expired(tw, p.spin_limit_ns)) {
                            set_error(p.ctr, GCC_ETIMEOUT, W_STARVE);
                            bad = 1;
                            break;
                        }
                        __nanosleep(1000);
                    }
                }
                if (g.bcast(bad, 0)) { st = kGiveUp; break; }
            }
            // After 8 failed attempts, a short random pause (up to
            // backoff_ns, at most a few microseconds) breaks the symmetric
            // retry patterns that lock-step warps can otherwise repeat
            // forever, e.g. two OCC transactions that each read what the
            // other writes and abort on each other's write lock. It is kept
            // short because a batch ends with its slowest transaction. The
            // commit rule is untouched.
            if (p.backoff_ns && attempts >= 8u)
                __nanosleep((unsigned)(hash3(tx, attempts, 0x5ull) % p.backoff_ns));
            c_abort += clock64() - c_attempt;
            if (g.any(expired(t_start, 4ull * p.spin_limit_ns) || error_raised(p.ctr))) {
                if (g.glane == 0) set_error(p.ctr, GCC_ETIMEOUT, W_RETRY);
                st = kGiveUp;
                break;
            }
        }
        if (starving && g.glane == 0) {
            atomicCAS(&p.ctr->starve_token, tx + 1u, 0u);
            atomicSub(&p.ctr->starving, 1u);
        }
        if (st == kGiveUp) break;
        dg = g.sum(dg);
        if (g.glane == 0) {
            const long long c_end = clock64();
            p.digest[tx] = dg;
            p.tx_aborts[tx] = attempts;
            if (attempts > 64) atomicMax(&p.ctr->max_attempts, attempts + 1u);
            atomicAdd(&s_met[0], 1ull);
            atomicAdd(&s_met[1], (unsigned long long)attempts);
            atomicAdd(&s_met[2], ck.ts);
            atomicAdd(&s_met[3], ck.wait);
            atomicAdd(&s_met[4], c_abort);
            atomicAdd(&s_met[5], (unsigned long long)(c_end - c_attempt));
            atomicAdd(&s_met[6], (unsigned long long)(c_end - c_start));
            atomicAdd(&s_met[7], (unsigned long long)(c_after_idx - c_start));
            atomicAdd(&s_hist[hist_bucket(gtimer() - t_start)], 1u);
        }
    }

    __syncthreads();
    if (threadIdx.x < 8 && s_met[threadIdx.x]) {
        Counters *c = p.ctr;
        unsigned long long *dst[8] = {&c->committed, &c->aborts, &c->ts_cycles, &c->wait_cycles,
                                      &c->abort_cycles, &c->mng_cycles, &c->tot_cycles,
                                      &c->idx_cycles};
        atomicAdd(dst[threadIdx.x], s_met[threadIdx.x]);
    }
    for (int i = threadIdx.x; i < kHistBuckets; i += blockDim.x)
        if (s_hist[i]) atomicAdd(&p.ctr->hist[i], s_hist[i]);
}

// Launch helper implemented once per scheme translation unit.
cudaError_t launch_scheme(int scheme, int G, int grid, int block, const KParams &p,
                          cudaStream_t stream);
int occupancy_blocks(int scheme, int G, int block);

}  // namespace gcc
