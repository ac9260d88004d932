// orderentry.cpp -- integer order-entry workload: row layout and request
// generator for new-order / payment transactions over the engine's u64 row
// table, in the variable-length request format with extended ops.
//
// Shape from the reference's TPC-C path (benchmark/tpcc.cu:35-380,
// generation/gen_tpcc.cu:108-182, include/tpcc.cuh): warehouses x districts x
// customers, an item catalogue and one stock row per (warehouse, item),
// new-order with 5-15 order lines whose items follow NURand(8191) and come
// from a remote warehouse with a small probability, payment with a remote
// customer share. Differences: money is integer cents (the reference uses
// floats), and the ids of the rows a transaction inserts are assigned at
// generation time (a slot per transaction in an insert area) so that every
// transaction is a static list of (row, op) requests; the district's
// next-order-id is still read and incremented by the transaction.
//
// Row groups (u64 key = row id, fields 0-9):
//   warehouse w               0 ytd (cents)       1 tax (basis points)
//   district  w*D + d         0 ytd               1 tax      2 next_o_id
//   customer  (w*D + d)*C + c 0 balance (signed)  1 ytd_payment
//                             2 payment_cnt       3 discount (bp)
//   item      i               0 price (cents)   (read only)
//   stock     w*I + i         0 quantity  1 ytd  2 order_cnt  3 remote_cnt
//   inserts                   order, order-line and history rows
// Requests of a transaction are sorted by row id (distinct rows).
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "../../include/gcc_engine.h"

namespace {

uint64_t splitmix64(uint64_t x) {
    uint64_t z = x + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
uint64_t hash3(uint64_t s, uint64_t a, uint64_t b) {
    return splitmix64(splitmix64(s ^ (a * 0x9E3779B97F4A7C15ull)) ^ (b * 0xC2B2AE3D27D4EB4Full));
}

struct Rng {
    uint64_t seed, tx, c = 0;
    uint64_t next() { return hash3(seed, tx, c++); }
    uint32_t uniform(uint32_t lo, uint32_t hi) {  // inclusive
        return lo + (uint32_t)(next() % (uint64_t)(hi - lo + 1));
    }
};

// NURand(A, x, y) of the order-entry specification, with the run constant c.
uint32_t nurand(Rng &r, uint32_t a, uint32_t x, uint32_t y, uint32_t c) {
    return (((r.uniform(0, a) | r.uniform(x, y)) + c) % (y - x + 1)) + x;
}

bool desc_ok(const gcc_oe_desc *d) {
    return d && d->warehouses >= 1 && d->warehouses <= 4096 && d->districts >= 1 &&
           d->districts <= 100 && d->customers >= 1 && d->customers <= 100000 &&
           d->items >= 16 && d->items <= (1u << 20) && d->new_order_pct <= 100 &&
           d->remote_line_permille <= 1000 && d->remote_customer_pct <= 100 &&
           d->min_lines >= 1 && d->max_lines >= d->min_lines && d->max_lines <= 20;
}

void layout_of(const gcc_oe_desc *d, uint64_t inserts, gcc_oe_layout *l) {
    const uint64_t W = d->warehouses, D = d->districts, C = d->customers, I = d->items;
    l->warehouse = 0;
    l->district = W;
    l->customer = l->district + W * D;
    l->item = l->customer + W * D * C;
    l->stock = l->item + I;
    l->inserts = l->stock + W * I;
    l->rows = l->inserts + inserts;
}

constexpr uint64_t kSalt = 0x4F45ull;  // order-entry draws

// Kind and order-line count of transaction t (pure functions of (seed, t)).
void shape(const gcc_oe_desc *d, uint64_t seed, uint64_t t, bool *new_order, uint32_t *lines) {
    Rng r{seed ^ kSalt, t};
    *new_order = r.uniform(0, 99) < d->new_order_pct;
    *lines = r.uniform(d->min_lines, d->max_lines);
}
uint32_t n_requests(bool new_order, uint32_t lines) { return new_order ? 4 + 3 * lines : 4; }
uint32_t n_inserts(bool new_order, uint32_t lines) { return new_order ? 1 + lines : 1; }

}  // namespace

extern "C" int gcc_oe_offsets(const gcc_oe_desc *d, uint64_t n_tx, uint64_t seed, uint32_t *tx_off,
                              gcc_oe_layout *lay) {
    if (!desc_ok(d) || !tx_off || !lay) return GCC_EINVAL;
    uint64_t acc = 0, ins = 0;
    for (uint64_t t = 0; t < n_tx; ++t) {
        bool no;
        uint32_t lines;
        shape(d, seed, t, &no, &lines);
        tx_off[t] = (uint32_t)acc;
        acc += n_requests(no, lines);
        ins += n_inserts(no, lines);
        if (acc > 0xFFFFFFFFull) return GCC_EINVAL;
    }
    tx_off[n_tx] = (uint32_t)acc;
    layout_of(d, ins, lay);
    if (lay->rows > 0xFFFFFFFFull) return GCC_EINVAL;
    return GCC_OK;
}

extern "C" int gcc_oe_gen(const gcc_oe_desc *d, uint64_t n_tx, uint64_t seed, int32_t threads,
                          const uint32_t *tx_off, gcc_ycsb_req *reqs, uint8_t *kind) {
    if (!desc_ok(d) || !tx_off || (!reqs && n_tx)) return GCC_EINVAL;
    // insert slots: a prefix sum over the transactions' shapes
    std::vector<uint64_t> ins_off(n_tx + 1, 0);
    for (uint64_t t = 0; t < n_tx; ++t) {
        bool no;
        uint32_t lines;
        shape(d, seed, t, &no, &lines);
        if (tx_off[t + 1] - tx_off[t] != n_requests(no, lines)) return GCC_EINVAL;
        ins_off[t + 1] = ins_off[t] + n_inserts(no, lines);
    }
    gcc_oe_layout L;
    layout_of(d, ins_off[n_tx], &L);
    const uint32_t W = d->warehouses, D = d->districts, C = d->customers, I = d->items;
    const uint32_t c_cust = (uint32_t)(hash3(seed, 0x43ull, 1) % 1024ull);
    const uint32_t c_item = (uint32_t)(hash3(seed, 0x43ull, 2) % 8192ull);
    auto work = [&](uint64_t lo, uint64_t hi) {
        std::vector<gcc_ycsb_req> v;
        std::vector<uint32_t> items;
        for (uint64_t t = lo; t < hi; ++t) {
            bool no;
            uint32_t lines;
            shape(d, seed, t, &no, &lines);
            Rng r{seed ^ kSalt ^ 0x5EEDull, t};
            v.clear();
            const uint32_t w = r.uniform(0, W - 1), dd = r.uniform(0, D - 1);
            const uint64_t ins = L.inserts + ins_off[t];
            auto req = [&](int32_t op, uint64_t row) { v.push_back({op, (uint32_t)row}); };
            if (no) {
                const uint32_t c = nurand(r, 1023, 1, C, c_cust) - 1;
                const uint64_t dist = L.district + (uint64_t)w * D + dd;
                const uint64_t cust = L.customer + ((uint64_t)w * D + dd) * C + c;
                req(1, L.warehouse + w);                          // read tax
                req(GCC_OP_WORD(GCC_OP_ADD, 2, 1), dist);         // next_o_id += 1
                req(1, cust);                                     // read discount
                items.clear();
                for (uint32_t k = 0; k < lines; ++k) {
                    uint32_t it = 0;
                    for (int tries = 0; tries < 64; ++tries) {
                        it = nurand(r, 8191, 1, I, c_item) - 1;
                        if (std::find(items.begin(), items.end(), it) == items.end()) break;
                    }
                    while (std::find(items.begin(), items.end(), it) != items.end()) it = (it + 1) % I;
                    items.push_back(it);
                    const bool remote = W > 1 && r.uniform(0, 999) < d->remote_line_permille;
                    uint32_t sw = w;
                    if (remote) {
                        sw = r.uniform(0, W - 2);
                        if (sw >= w) ++sw;
                    }
                    const uint32_t qty = r.uniform(1, 10);
                    req(1, L.item + it);                          // read price
                    req(GCC_OP_WORD(GCC_OP_STOCK, 0, qty | (remote ? 0x100u : 0u)),
                        L.stock + (uint64_t)sw * I + it);
                    req(GCC_OP_WORD(GCC_OP_INSERT, 0, (it & 0x1FFFFu) | (qty << 17)),
                        ins + 1 + k);                             // order line
                }
                req(GCC_OP_WORD(GCC_OP_INSERT, 0, (dd * C + c) & 0xFFFFFFu), ins);  // order
            } else {
                uint32_t cw = w, cd = dd;
                if (W > 1 && r.uniform(0, 99) < d->remote_customer_pct) {
                    cw = r.uniform(0, W - 2);
                    if (cw >= w) ++cw;
                    cd = r.uniform(0, D - 1);
                }
                const uint32_t c = nurand(r, 1023, 1, C, c_cust) - 1;
                const uint32_t amount = r.uniform(1, 5000);
                req(GCC_OP_WORD(GCC_OP_ADD, 0, amount), L.warehouse + w);                      // w ytd
                req(GCC_OP_WORD(GCC_OP_ADD, 0, amount), L.district + (uint64_t)w * D + dd);   // d ytd
                req(GCC_OP_WORD(GCC_OP_PAY, 0, amount),
                    L.customer + ((uint64_t)cw * D + cd) * C + c);
                req(GCC_OP_WORD(GCC_OP_INSERT, 0, amount), ins);                              // history
            }
            std::sort(v.begin(), v.end(),
                      [](const gcc_ycsb_req &a, const gcc_ycsb_req &b) { return a.key < b.key; });
            memcpy(reqs + tx_off[t], v.data(), v.size() * sizeof(gcc_ycsb_req));
            if (kind) kind[t] = no ? 1 : 2;
        }
    };
    unsigned nt = threads > 0 ? (unsigned)threads : std::max(1u, std::thread::hardware_concurrency());
    if ((uint64_t)nt > n_tx) nt = (unsigned)std::max<uint64_t>(1, n_tx);
    std::vector<std::thread> pool;
    const uint64_t per = (n_tx + nt - 1) / nt;
    for (unsigned i = 0; i < nt; ++i) {
        const uint64_t lo = (uint64_t)i * per, hi = std::min<uint64_t>(n_tx, lo + per);
        if (lo >= hi) break;
        pool.emplace_back(work, lo, hi);
    }
    for (auto &th : pool) th.join();
    return GCC_OK;
}
