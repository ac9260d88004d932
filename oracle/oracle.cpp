// oracle.cpp -- CPU oracle of the YCSB transaction path (test infrastructure;
// see oracle.h). Written independently of the engine: the value formulas
// below are restated from their definition, not included from the engine.
#include "oracle.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <thread>
#include <vector>

namespace {

// ---- value formulas (definition shared with the engine, restated) --------
uint64_t sm64(uint64_t x) {
    uint64_t z = x + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
uint64_t h3(uint64_t s, uint64_t a, uint64_t b) {
    return sm64(sm64(s ^ (a * 0x9E3779B97F4A7C15ull)) ^ (b * 0xC2B2AE3D27D4EB4Full));
}
uint64_t term(uint64_t word, uint32_t op, uint32_t k) {
    return sm64(word ^ ((uint64_t)(op * 16u + k + 1u) * 0xD6E8FEB86659FD93ull));
}
uint32_t rbytes(int32_t layout) { return layout == GCC_LAYOUT_REF104 ? 104u : 88u; }
uint32_t rstride(int32_t layout) { return layout == GCC_LAYOUT_REF104 ? 112u : 96u; }

uint64_t load_word(const uint8_t *p) {
    uint64_t v;
    memcpy(&v, p, 8);
    return v;
}
void store_word(uint8_t *p, uint64_t v) { memcpy(p, &v, 8); }

// Extended write op (request `read` < 0, gcc_engine.h GCC_OP_*) on a packed
// u64 row of `words` words: returns the digest term of the row image it
// reads (read-modify-writes) or 0 (insert); GCC_EFORMAT via *bad.
uint64_t ext_op(uint8_t *r, uint32_t words, uint32_t w, uint64_t wseed, uint32_t tx, uint32_t i,
                bool *bad) {
    const uint32_t op = (w >> 28) & 7u, f = (w >> 24) & 15u, v = w & 0xFFFFFFu;
    const uint32_t fmax = op == GCC_OP_STOCK ? 6u : (op == GCC_OP_PAY ? 7u : 9u);
    if (op < GCC_OP_ADD || op > GCC_OP_INSERT || f > fmax || words != 11u) {
        *bad = true;
        return 0;
    }
    auto fld = [&](uint32_t k) { return r + 8 * (1 + k); };
    if (op == GCC_OP_INSERT) {
        store_word(fld(0), tx);
        store_word(fld(1), v);
        for (uint32_t k = 0; k < 8; ++k) store_word(fld(2 + k), h3(wseed, tx, 1024ull + i * 8ull + k));
        return 0;
    }
    uint64_t dt = 0;
    for (uint32_t k = 0; k < words; ++k) dt += term(load_word(r + 8 * k), i, k);
    const uint64_t a = load_word(fld(f));
    switch (op) {
        case GCC_OP_ADD: store_word(fld(f), a + v); break;
        case GCC_OP_SUB: store_word(fld(f), a - v); break;
        case GCC_OP_STOCK: {
            const uint64_t q = v & 0xFFu, remote = (v >> 8) & 1u;
            store_word(fld(f), a >= q + 10 ? a - q : a - q + 91);
            store_word(fld(f + 1), load_word(fld(f + 1)) + q);
            store_word(fld(f + 2), load_word(fld(f + 2)) + 1);
            store_word(fld(f + 3), load_word(fld(f + 3)) + remote);
            break;
        }
        case GCC_OP_PAY:
            store_word(fld(f), a - v);
            store_word(fld(f + 1), load_word(fld(f + 1)) + v);
            store_word(fld(f + 2), load_word(fld(f + 2)) + 1);
            break;
    }
    return dt;
}

struct Ctx {
    uint8_t *table;
    uint64_t rows;
    int32_t layout;
    uint32_t rb, words;
    int32_t write_mode;
    uint64_t wseed;
};

// One YCSB transaction in program order (benchmark/ycsb.cu:57-98): `item` is
// the transaction-local row buffer, zero at start; a read copies the row
// into it; a write stores a field value or copies `item` over the row.
int run_serial(const Ctx &c, const gcc_ycsb_tx &tx, uint32_t txid, uint64_t *digest,
               uint8_t *read_log) {
    if (tx.request_cnt > 16) return GCC_EFORMAT;
    std::vector<uint8_t> item(c.rb, 0);
    uint64_t dg = 0;
    for (uint32_t i = 0; i < tx.request_cnt; ++i) {
        const gcc_ycsb_req &rq = tx.requests[i];
        uint64_t row = rq.key;  // keys are row ids (row r holds key r)
        if (row >= c.rows) return GCC_EKEY;
        uint8_t *r = c.table + row * c.rb;
        if (rq.read > 0) {
            for (uint32_t k = 0; k < c.words; ++k) dg += term(load_word(r + 8 * k), i, k);
            memcpy(item.data(), r, c.rb);
            if (read_log) memcpy(read_log + ((uint64_t)txid * 16 + i) * rstride(c.layout), r, c.rb);
        } else if (c.write_mode == GCC_WRITE_FIELD) {
            uint32_t f = (uint32_t)(h3(c.wseed, txid, 2ull * i) % 10ull);
            store_word(r + 8 * (1 + f), h3(c.wseed, txid, 2ull * i + 1));
        } else {
            memcpy(r, item.data(), c.rb);
        }
    }
    if (digest) digest[txid] = dg;
    return GCC_OK;
}

}  // namespace

extern "C" {

int oracle_fill_table(uint64_t rows, int32_t layout, uint64_t seed, uint8_t *out) {
    const uint32_t rb = rbytes(layout), words = rb / 8;
    for (uint64_t r = 0; r < rows; ++r) {
        for (uint32_t k = 0; k < words; ++k) {
            uint64_t v = seed ? h3(seed, r, k) : 0;
            if (k == 0) v = layout == GCC_LAYOUT_U64X11 ? r : ((v & 0xFFFFFFFF00000000ull) | (uint32_t)r);
            store_word(out + r * rb + 8 * k, v);
        }
    }
    return GCC_OK;
}

int oracle_replay_var(uint8_t *table, uint64_t rows, int32_t layout, const uint32_t *tx_off,
                      const gcc_ycsb_req *reqs, uint64_t n_tx, const uint32_t *order,
                      uint64_t n_order, int32_t write_mode, uint64_t write_seed,
                      uint64_t *digests) {
    return oracle_replay_var_ext(table, rows, layout, tx_off, reqs, n_tx, order, n_order,
                                 write_mode, write_seed, digests, 0);
}

int oracle_replay_var_ext(uint8_t *table, uint64_t rows, int32_t layout, const uint32_t *tx_off,
                          const gcc_ycsb_req *reqs, uint64_t n_tx, const uint32_t *order,
                          uint64_t n_order, int32_t write_mode, uint64_t write_seed,
                          uint64_t *digests, int32_t ext_ops) {
    Ctx c{table, rows, layout, rbytes(layout), rbytes(layout) / 8, write_mode, write_seed};
    std::vector<uint8_t> item(c.rb);
    for (uint64_t j = 0; j < n_order; ++j) {
        uint32_t t = order ? order[j] : (uint32_t)j;
        if (t >= n_tx) return GCC_EINVAL;
        uint32_t n = tx_off[t + 1] - tx_off[t];
        if (n > 64) return GCC_EFORMAT;
        std::fill(item.begin(), item.end(), 0);
        uint64_t dg = 0;
        for (uint32_t i = 0; i < n; ++i) {
            const gcc_ycsb_req &rq = reqs[tx_off[t] + i];
            if (rq.key >= rows) return GCC_EKEY;
            uint8_t *r = c.table + (uint64_t)rq.key * c.rb;
            if (rq.read > 0) {
                for (uint32_t k = 0; k < c.words; ++k) dg += term(load_word(r + 8 * k), i, k);
                memcpy(item.data(), r, c.rb);
            } else if (ext_ops && rq.read < 0) {
                bool bad = false;
                dg += ext_op(r, c.words, (uint32_t)rq.read, c.wseed, t, i, &bad);
                if (bad) return GCC_EFORMAT;
            } else if (c.write_mode == GCC_WRITE_FIELD) {
                uint32_t f = (uint32_t)(h3(c.wseed, t, 2ull * i) % 10ull);
                store_word(r + 8 * (1 + f), h3(c.wseed, t, 2ull * i + 1));
            } else {
                memcpy(r, item.data(), c.rb);
            }
        }
        if (digests) digests[t] = dg;
    }
    return GCC_OK;
}

int oracle_replay(uint8_t *table, uint64_t rows, int32_t layout, const gcc_ycsb_tx *txs,
                  uint64_t n_tx, const uint32_t *order, uint64_t n_order, int32_t write_mode,
                  uint64_t write_seed, uint64_t *digests, uint8_t *read_log) {
    Ctx c{table, rows, layout, rbytes(layout), rbytes(layout) / 8, write_mode, write_seed};
    for (uint64_t j = 0; j < n_order; ++j) {
        uint32_t t = order ? order[j] : (uint32_t)j;
        if (t >= n_tx) return GCC_EINVAL;
        int rc = run_serial(c, txs[t], t, digests, read_log);
        if (rc) return rc;
    }
    return GCC_OK;
}

// Rank function of gputx_pre2 (src/gputx.cu:17-27): walk each object's
// accesses in ascending tx order; an access gets the current rank, and the
// rank grows after any pair that is not read/read. A tx's rank is the max
// over its accesses. (The reference's last object reads offset[dense_cnt],
// past the scanned counts; here every object's list ends at its last access.)
int oracle_gputx_order(const gcc_ycsb_tx *txs, uint64_t n_tx, uint64_t rows, uint32_t *ranks,
                       uint32_t *order, uint32_t *max_rank) {
    std::map<uint32_t, std::vector<std::pair<uint32_t, bool>>> lists;
    for (uint64_t t = 0; t < n_tx; ++t) {
        if (txs[t].request_cnt > 16) return GCC_EFORMAT;
        for (uint32_t i = 0; i < txs[t].request_cnt; ++i) {
            uint32_t key = txs[t].requests[i].key;
            if (key >= rows) return GCC_EKEY;
            lists[key].push_back({(uint32_t)t, txs[t].requests[i].read != 0});
        }
    }
    std::vector<uint32_t> rk(n_tx, 0);
    uint32_t mx = 0;
    for (auto &kv : lists) {
        auto &l = kv.second;  // already in ascending tx order
        uint32_t cur = 0;
        for (size_t i = 0; i < l.size(); ++i) {
            rk[l[i].first] = std::max(rk[l[i].first], cur);
            mx = std::max(mx, cur);
            if (i + 1 < l.size() && (!l[i].second || !l[i + 1].second)) ++cur;
        }
    }
    std::vector<uint32_t> ord(n_tx);
    for (uint64_t t = 0; t < n_tx; ++t) ord[t] = (uint32_t)t;
    std::stable_sort(ord.begin(), ord.end(), [&](uint32_t a, uint32_t b) { return rk[a] < rk[b]; });
    if (ranks) memcpy(ranks, rk.data(), n_tx * 4);
    if (order) memcpy(order, ord.data(), n_tx * 4);
    if (max_rank) *max_rank = mx;
    return GCC_OK;
}

int oracle_commit_order(const gcc_commit_rec *log, uint64_t n_tx, uint32_t *order) {
    std::vector<uint32_t> ord(n_tx);
    for (uint64_t t = 0; t < n_tx; ++t) ord[t] = (uint32_t)t;
    std::sort(ord.begin(), ord.end(), [&](uint32_t a, uint32_t b) {
        if (log[a].hi != log[b].hi) return log[a].hi < log[b].hi;
        if (log[a].lo != log[b].lo) return log[a].lo < log[b].lo;
        return a < b;
    });
    memcpy(order, ord.data(), n_tx * 4);
    return GCC_OK;
}

// Edges of ExecInfo::scan_events (src/runtime.cu:23-71): over events in seq
// order, a read of o by T depends on every other active tx that wrote o; a
// write of o by T depends on every other active accessor of o; a tx leaves
// the active sets of its objects when its commit event (is_write == 2) is
// seen. Cycle search by iterative DFS (src/runtime.cu:80-98).
int oracle_conflict_acyclic(const oracle_event *ev, uint64_t n_ev, uint64_t n_tx) {
    std::vector<const oracle_event *> es(n_ev);
    for (uint64_t i = 0; i < n_ev; ++i) es[i] = ev + i;
    std::stable_sort(es.begin(), es.end(),
                     [](const oracle_event *a, const oracle_event *b) { return a->seq < b->seq; });
    std::map<uint32_t, std::map<uint32_t, bool>> active;  // row -> tx -> wrote
    std::vector<std::vector<uint32_t>> ops(n_tx);
    std::vector<std::vector<uint32_t>> graph(n_tx);
    for (const oracle_event *e : es) {
        if (e->tx >= n_tx) return 0;
        if (e->is_write == 2) {
            for (uint32_t o : ops[e->tx]) active[o].erase(e->tx);
            continue;
        }
        ops[e->tx].push_back(e->row);
        auto &act = active[e->row];
        for (auto &kv : act) {
            if (kv.first == e->tx) continue;
            if (e->is_write || kv.second) graph[e->tx].push_back(kv.first);
        }
        act[e->tx] = act[e->tx] || e->is_write;
    }
    std::vector<uint8_t> color(n_tx, 0);
    std::vector<std::pair<uint32_t, size_t>> st;
    for (uint64_t s = 0; s < n_tx; ++s) {
        if (color[s]) continue;
        st.push_back({(uint32_t)s, 0});
        color[s] = 1;
        while (!st.empty()) {
            auto &top = st.back();
            if (top.second < graph[top.first].size()) {
                uint32_t nx = graph[top.first][top.second++];
                if (color[nx] == 1) return 0;
                if (color[nx] == 0) {
                    color[nx] = 1;
                    st.push_back({nx, 0});
                }
            } else {
                color[top.first] = 2;
                st.pop_back();
            }
        }
    }
    return 1;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Multi-threaded CPU executors (baseline). Metadata words follow the same
// commit rules as the GPU schemes: 2PL no-wait (twopl.cuh:233-303), Silo
// (silo.cuh:223-338), TicToc (tictoc.cuh:223-368). Row words are accessed
// with relaxed 64-bit atomics; lock/ts words with acq/rel atomics.
// ---------------------------------------------------------------------------
namespace {

struct Cpu {
    uint8_t *table;
    uint64_t rows;
    uint32_t rb, words;
    int32_t write_mode;
    uint64_t wseed;
    bool ext = false;  // negative read words are extended ops
    std::atomic<uint64_t> *meta;
    std::atomic<uint64_t> seq{0};
    // transactions: 16-request records, or CSR (tx_off, reqs)
    const gcc_ycsb_tx *txs = nullptr;
    const uint32_t *tx_off = nullptr;
    const gcc_ycsb_req *reqs = nullptr;
    uint64_t n_tx;
    uint64_t *digests;
    gcc_commit_rec *log;

    uint32_t n_req(uint32_t t) const {
        return txs ? (uint32_t)txs[t].request_cnt : tx_off[t + 1] - tx_off[t];
    }
    const gcc_ycsb_req &req(uint32_t t, uint32_t i) const {
        return txs ? txs[t].requests[i] : reqs[tx_off[t] + i];
    }
    bool is_read(uint32_t t, uint32_t i) const { return req(t, i).read > 0; }
    uint64_t *rowp(uint64_t r) const { return (uint64_t *)(table + r * rb); }
    uint64_t ld(const uint64_t *p) const { return __atomic_load_n(p, __ATOMIC_RELAXED); }
    void st(uint64_t *p, uint64_t v) const { __atomic_store_n(p, v, __ATOMIC_RELAXED); }
    uint64_t read_row(uint64_t r, uint32_t i, uint64_t *img) const {
        uint64_t d = 0;
        const uint64_t *p = rowp(r);
        for (uint32_t k = 0; k < words; ++k) {
            img[k] = ld(p + k);
            d += term(img[k], i, k);
        }
        return d;
    }
    // Extended op on a row held exclusively (same rules as ext_op above,
    // with the executors' atomic word accesses); returns its digest term.
    uint64_t ext_write(uint64_t r, uint32_t tx, uint32_t i, uint32_t w) const {
        uint64_t *p = rowp(r);
        const uint32_t op = (w >> 28) & 7u, f = (w >> 24) & 15u, v = w & 0xFFFFFFu;
        if (op == GCC_OP_INSERT) {
            st(p + 1, tx);
            st(p + 2, v);
            for (uint32_t k = 0; k < 8; ++k) st(p + 3 + k, h3(wseed, tx, 1024ull + i * 8ull + k));
            return 0;
        }
        uint64_t dt = 0;
        for (uint32_t k = 0; k < words; ++k) dt += term(ld(p + k), i, k);
        uint64_t *fw = p + 1 + f;
        const uint64_t a = ld(fw);
        if (op == GCC_OP_ADD) st(fw, a + v);
        else if (op == GCC_OP_SUB) st(fw, a - v);
        else if (op == GCC_OP_STOCK) {
            const uint64_t q = v & 0xFFu, remote = (v >> 8) & 1u;
            st(fw, a >= q + 10 ? a - q : a - q + 91);
            st(fw + 1, ld(fw + 1) + q);
            st(fw + 2, ld(fw + 2) + 1);
            st(fw + 3, ld(fw + 3) + remote);
        } else if (op == GCC_OP_PAY) {
            st(fw, a - v);
            st(fw + 1, ld(fw + 1) + v);
            st(fw + 2, ld(fw + 2) + 1);
        }
        return dt;
    }
    // write request i of tx (field write, row copy, or extended op)
    uint64_t write_op(uint32_t tx, uint32_t i, const uint64_t *item) const {
        const gcc_ycsb_req &rq = req(tx, i);
        if (ext && rq.read < 0) return ext_write(rq.key, tx, i, (uint32_t)rq.read);
        uint64_t *p = rowp(rq.key);
        if (write_mode == GCC_WRITE_FIELD) {
            uint32_t f = (uint32_t)(h3(wseed, tx, 2ull * i) % 10ull);
            st(p + 1 + f, h3(wseed, tx, 2ull * i + 1));
        } else {
            for (uint32_t k = 0; k < words; ++k) st(p + k, item[k]);
        }
        return 0;
    }
};

constexpr uint64_t kExcl = 1ull << 31;
constexpr uint64_t kLock = 1ull << 63;
constexpr uint32_t kCpuMaxReq = 64;

// Source image for a rowcopy write: the last read before op i.
const uint64_t *src_image(const Cpu &c, uint32_t t, uint32_t i, const std::vector<uint64_t> &imgs,
                          const std::vector<uint64_t> &zero) {
    for (int j = (int)i - 1; j >= 0; --j)
        if (c.is_read(t, (uint32_t)j)) return imgs.data() + (size_t)j * c.words;
    return zero.data();
}

bool tx_tpl_nw(Cpu &c, uint32_t t, std::vector<uint64_t> &imgs, const std::vector<uint64_t> &zero) {
    const uint32_t n = c.n_req(t);
    uint32_t held = 0;
    for (uint32_t i = 0; i < n; ++i) {
        std::atomic<uint64_t> &m = c.meta[c.req(t, i).key];
        bool ok;
        if (c.is_read(t, i)) {
            uint64_t old = m.fetch_add(1, std::memory_order_acq_rel);
            ok = !(old & kExcl);
            if (!ok) m.fetch_sub(1, std::memory_order_acq_rel);
        } else {
            uint64_t exp = 0;
            ok = m.compare_exchange_strong(exp, kExcl | ((uint64_t)t << 32), std::memory_order_acq_rel);
        }
        if (!ok) {
            for (uint32_t j = 0; j < held; ++j) {
                std::atomic<uint64_t> &mj = c.meta[c.req(t, j).key];
                if (c.is_read(t, j)) mj.fetch_sub(1, std::memory_order_acq_rel);
                else mj.fetch_and(0x7FFFFFFFull, std::memory_order_acq_rel);
            }
            return false;
        }
        held = i + 1;
    }
    if (c.log) c.log[t] = gcc_commit_rec{c.seq.fetch_add(1), 0};
    uint64_t dg = 0;
    for (uint32_t i = 0; i < n; ++i)
        if (c.is_read(t, i)) dg += c.read_row(c.req(t, i).key, i, imgs.data() + (size_t)i * c.words);
    for (uint32_t i = 0; i < n; ++i)
        if (!c.is_read(t, i)) dg += c.write_op(t, i, src_image(c, t, i, imgs, zero));
    for (uint32_t i = 0; i < n; ++i) {
        std::atomic<uint64_t> &m = c.meta[c.req(t, i).key];
        if (c.is_read(t, i)) m.fetch_sub(1, std::memory_order_acq_rel);
        else m.fetch_and(0x7FFFFFFFull, std::memory_order_acq_rel);
    }
    c.digests[t] = dg;
    return true;
}

template <bool TICTOC>
bool tx_occ(Cpu &c, uint32_t t, std::vector<uint64_t> &imgs, const std::vector<uint64_t> &zero) {
    const uint32_t n = c.n_req(t);
    uint64_t rec[kCpuMaxReq], dg = 0;
    const uint64_t wmask = (1ull << 48) - 1;
    for (uint32_t i = 0; i < n; ++i) {
        if (!c.is_read(t, i)) continue;
        std::atomic<uint64_t> &m = c.meta[c.req(t, i).key];
        while (true) {
            uint64_t x1 = m.load(std::memory_order_acquire);
            if (x1 & kLock) continue;
            uint64_t d = c.read_row(c.req(t, i).key, i, imgs.data() + (size_t)i * c.words);
            std::atomic_thread_fence(std::memory_order_acquire);
            if (m.load(std::memory_order_acquire) != x1) continue;
            rec[i] = x1;
            dg += d;
            break;
        }
    }
    uint64_t locked = 0;
    uint64_t cts = 0;
    bool fail = false;
    for (uint32_t i = 0; i < n && !fail; ++i) {
        if (c.is_read(t, i)) continue;
        std::atomic<uint64_t> &m = c.meta[c.req(t, i).key];
        uint64_t x = m.load(std::memory_order_acquire);
        while (true) {
            if (x & kLock) { fail = true; break; }
            if (m.compare_exchange_weak(x, x | kLock, std::memory_order_acq_rel)) break;
        }
        if (fail) break;
        locked |= 1ull << i;
        uint64_t c1 = TICTOC ? (x & wmask) + ((x >> 48) & 0x7FFF) + 1 : (x & ~kLock);
        cts = std::max(cts, c1);
    }
    uint64_t seqv = 0;
    if (!fail && !TICTOC && c.log) seqv = c.seq.fetch_add(1);
    if (!fail) {
        if (!TICTOC) {
            for (uint32_t i = 0; i < n && !fail; ++i) {
                if (!c.is_read(t, i)) continue;
                uint64_t x = c.meta[c.req(t, i).key].load(std::memory_order_acquire);
                if (x != rec[i]) fail = true;  // ts changed or locked
                cts = std::max(cts, rec[i] & ~kLock);
            }
            cts += 1;
        } else {
            for (uint32_t i = 0; i < n; ++i)
                if (c.is_read(t, i)) cts = std::max(cts, rec[i] & wmask);
            for (uint32_t i = 0; i < n && !fail; ++i) {
                if (!c.is_read(t, i)) continue;
                uint64_t rwts = rec[i] & wmask, rrts = rwts + ((rec[i] >> 48) & 0x7FFF);
                if (rrts >= cts) continue;
                std::atomic<uint64_t> &m = c.meta[c.req(t, i).key];
                while (true) {
                    uint64_t x = m.load(std::memory_order_acquire);
                    uint64_t wts = x & wmask, rts = wts + ((x >> 48) & 0x7FFF);
                    if (wts != rwts || (rts <= cts && (x & kLock))) { fail = true; break; }
                    if (rts > cts) break;
                    uint64_t delta = cts - wts, shift = delta - (delta & 0x7FFF);
                    uint64_t nx = ((delta - shift) << 48) | ((wts + shift) & wmask);
                    if (m.compare_exchange_weak(x, nx, std::memory_order_acq_rel)) break;
                }
            }
            if (!fail && c.log) seqv = c.seq.fetch_add(1);
        }
    }
    if (fail) {
        for (uint32_t i = 0; i < n; ++i)
            if ((locked >> i) & 1ull) c.meta[c.req(t, i).key].fetch_and(~kLock, std::memory_order_acq_rel);
        return false;
    }
    for (uint32_t i = 0; i < n; ++i)
        if (!c.is_read(t, i)) dg += c.write_op(t, i, src_image(c, t, i, imgs, zero));
    for (uint32_t i = 0; i < n; ++i)
        if (!c.is_read(t, i))
            c.meta[c.req(t, i).key].store(TICTOC ? (cts & wmask) : cts, std::memory_order_release);
    if (c.log) c.log[t] = TICTOC ? gcc_commit_rec{cts, seqv} : gcc_commit_rec{seqv, 0};
    c.digests[t] = dg;
    return true;
}

// The executor loop shared by both record formats.
int cpu_execute(Cpu &c, int kind, int32_t threads, double *seconds, uint64_t *aborts) {
    std::vector<std::atomic<uint64_t>> meta(c.rows);
    for (auto &m : meta) m.store(0, std::memory_order_relaxed);
    c.meta = meta.data();
    const uint64_t n_tx = c.n_tx;
    unsigned nt = threads > 0 ? (unsigned)threads : std::max(1u, std::thread::hardware_concurrency());
    std::atomic<uint64_t> next{0}, ab{0};
    auto t0 = std::chrono::steady_clock::now();
    auto worker = [&]() {
        std::vector<uint64_t> imgs((size_t)kCpuMaxReq * c.words), zero(c.words, 0);
        uint64_t my_ab = 0;
        while (true) {
            uint64_t t = next.fetch_add(1);
            if (t >= n_tx) break;
            while (true) {
                bool ok = kind == 0 ? tx_tpl_nw(c, (uint32_t)t, imgs, zero)
                        : kind == 1 ? tx_occ<false>(c, (uint32_t)t, imgs, zero)
                                    : tx_occ<true>(c, (uint32_t)t, imgs, zero);
                if (ok) break;
                ++my_ab;
                std::this_thread::yield();
            }
        }
        ab += my_ab;
    };
    std::vector<std::thread> pool;
    for (unsigned i = 0; i < nt; ++i) pool.emplace_back(worker);
    for (auto &th : pool) th.join();
    auto t1 = std::chrono::steady_clock::now();
    if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
    if (aborts) *aborts = ab.load();
    return GCC_OK;
}

int scheme_kind(const char *scheme) {
    std::string s = scheme ? scheme : "";
    return s == "tpl_nw" ? 0 : s == "silo" ? 1 : s == "tictoc" ? 2 : -1;
}

}  // namespace

extern "C" int oracle_cpu_run(const char *scheme, uint8_t *table, uint64_t rows, int32_t layout,
                              const gcc_ycsb_tx *txs, uint64_t n_tx, int32_t write_mode,
                              uint64_t write_seed, int32_t threads, uint64_t *digests,
                              gcc_commit_rec *commit_log, double *seconds, uint64_t *aborts) {
    const int kind = scheme_kind(scheme);
    if (kind < 0 || !table || !digests) return GCC_EINVAL;
    for (uint64_t t = 0; t < n_tx; ++t) {
        if (txs[t].request_cnt > 16) return GCC_EFORMAT;
        for (uint32_t i = 0; i < txs[t].request_cnt; ++i)
            if (txs[t].requests[i].key >= rows) return GCC_EKEY;
    }
    Cpu c;
    c.table = table;
    c.rows = rows;
    c.rb = rbytes(layout);
    c.words = c.rb / 8;
    c.write_mode = write_mode;
    c.wseed = write_seed;
    c.txs = txs;
    c.n_tx = n_tx;
    c.digests = digests;
    c.log = commit_log;
    return cpu_execute(c, kind, threads, seconds, aborts);
}

extern "C" int oracle_cpu_run_var(const char *scheme, uint8_t *table, uint64_t rows,
                                  int32_t layout, const uint32_t *tx_off,
                                  const gcc_ycsb_req *reqs, uint64_t n_tx, int32_t write_mode,
                                  uint64_t write_seed, int32_t ext_ops, int32_t threads,
                                  uint64_t *digests, gcc_commit_rec *commit_log, double *seconds,
                                  uint64_t *aborts) {
    const int kind = scheme_kind(scheme);
    if (kind < 0 || !table || !digests || !tx_off || (!reqs && n_tx)) return GCC_EINVAL;
    const uint32_t words = rbytes(layout) / 8;
    for (uint64_t t = 0; t < n_tx; ++t) {
        if (tx_off[t + 1] < tx_off[t] || tx_off[t + 1] - tx_off[t] > kCpuMaxReq) return GCC_EFORMAT;
        for (uint32_t i = tx_off[t]; i < tx_off[t + 1]; ++i) {
            if (reqs[i].key >= rows) return GCC_EKEY;
            if (ext_ops && reqs[i].read < 0) {
                const uint32_t w = (uint32_t)reqs[i].read, op = (w >> 28) & 7u, f = (w >> 24) & 15u;
                const uint32_t fmax = op == GCC_OP_STOCK ? 6u : (op == GCC_OP_PAY ? 7u : 9u);
                if (op < GCC_OP_ADD || op > GCC_OP_INSERT || f > fmax || words != 11u)
                    return GCC_EFORMAT;
            }
        }
    }
    Cpu c;
    c.table = table;
    c.rows = rows;
    c.rb = rbytes(layout);
    c.words = words;
    c.write_mode = write_mode;
    c.wseed = write_seed;
    c.ext = ext_ops != 0;
    c.tx_off = tx_off;
    c.reqs = reqs;
    c.n_tx = n_tx;
    c.digests = digests;
    c.log = commit_log;
    return cpu_execute(c, kind, threads, seconds, aborts);
}

// Generator restated from generation/gen_ycsb.cu:76-152 (see oracle.h); the
// random stream is the same counter-based hash the engine's generator uses.
extern "C" int oracle_gen_ycsb(uint64_t rows, uint64_t n_tx, double theta, double read_ratio,
                               uint64_t seed, int32_t dedup, int32_t key_base, gcc_ycsb_tx *out) {
    if (rows < 3 || theta < 0 || theta >= 1.0) return GCC_EINVAL;
    const uint64_t n = key_base == 1 ? rows - 1 : rows;
    double zetan = 0;
    for (uint64_t i = 1; i <= n; ++i) zetan += std::pow(1.0 / (double)i, theta);
    const double zeta2 = 1.0 + std::pow(0.5, theta);
    const double alpha = 1.0 / (1.0 - theta);
    const double eta = (1.0 - std::pow(2.0 / (double)n, 1.0 - theta)) / (1.0 - zeta2 / zetan);
    auto uni = [&](uint64_t t, uint64_t c) {
        return (double)(h3(seed ^ 0x59435342ull, t, c) >> 11) * (1.0 / 9007199254740992.0);
    };
    for (uint64_t t = 0; t < n_tx; ++t) {
        gcc_ycsb_tx &tx = out[t];
        memset(&tx, 0, sizeof(tx));
        uint64_t c = 0;
        int rid = 0;
        int slots = dedup == GCC_DEDUP_DROP ? 16 : 16 * 1024;
        for (int slot = 0; slot < slots && rid < 16; ++slot) {
            double r = uni(t, c++);
            double u = uni(t, c++);
            double uz = u * zetan;
            uint64_t rank;
            if (uz < 1.0) rank = 1;
            else if (uz < 1.0 + std::pow(0.5, theta)) rank = 2;
            else {
                rank = 1 + (uint64_t)((double)n * std::pow(eta * u - eta + 1.0, alpha));
                if (rank > n) rank = n;
            }
            uint32_t key = (uint32_t)(key_base == 1 ? rank : rank - 1);
            bool dup = false;
            for (int j = 0; j < rid; ++j) dup |= tx.requests[j].key == key;
            if (dup) continue;
            tx.requests[rid].read = r < read_ratio ? 1 : 0;
            tx.requests[rid].key = key;
            ++rid;
        }
        tx.request_cnt = (uint64_t)rid;
        // ascending key order (the reference's bubble sort, gen_ycsb.cu:143-150)
        for (int i = rid - 1; i > 0; --i)
            for (int j = 0; j < i; ++j)
                if (tx.requests[j].key > tx.requests[j + 1].key) std::swap(tx.requests[j], tx.requests[j + 1]);
    }
    return GCC_OK;
}
