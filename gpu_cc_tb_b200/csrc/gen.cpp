// gen.cpp -- YCSB dataset generator writing gCCTB's raw YCSBTx records.
//
// Follows generation/gen_ycsb.cu:76-152 of the reference:
//   * Zipfian keys by the method of Gray et al., "Quickly generating
//     billion-record synthetic databases" (SIGMOD 1994), with
//     zetan = zeta(rows - 1, theta) and n = rows - 1, giving keys in
//     [1, rows - 1] (key_base 1), or shifted to [0, rows - 1] (key_base 0);
//   * each of the 16 request slots is a read with probability read_ratio;
//   * a repeated key is dropped (GCC_DEDUP_DROP, the reference) or redrawn
//     (GCC_DEDUP_RESAMPLE, exactly 16 distinct keys);
//   * requests are sorted by ascending key.
// Unlike the reference (256 threads sharing rand()), every draw is a counter-
// based hash of (seed, tx, draw), so the dataset is reproducible and the
// thread count does not change it.
#include <algorithm>
#include <cmath>
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
// Uniform double in [0, 1) from draw c of transaction tx.
double uniform(uint64_t seed, uint64_t tx, uint64_t c) {
    return (double)(hash3(seed ^ 0x59435342ull, tx, c) >> 11) * (1.0 / 9007199254740992.0);
}

struct Zipf {
    uint64_t n;
    double theta, zetan, zeta2, alpha, eta, half_pow;
    Zipf(uint64_t n_, double th) : n(n_), theta(th) {
        zetan = 0;
        for (uint64_t i = 1; i <= n; ++i) zetan += std::pow(1.0 / (double)i, theta);
        zeta2 = 1.0 + std::pow(0.5, theta);
        alpha = 1.0 / (1.0 - theta);
        eta = (1.0 - std::pow(2.0 / (double)n, 1.0 - theta)) / (1.0 - zeta2 / zetan);
        half_pow = std::pow(0.5, theta);
    }
    // rank in [1, n]
    uint64_t draw(double u) const {
        double uz = u * zetan;
        if (uz < 1.0) return 1;
        if (uz < 1.0 + half_pow) return 2;
        uint64_t r = 1 + (uint64_t)((double)n * std::pow(eta * u - eta + 1.0, alpha));
        return r > n ? n : r;
    }
};

}  // namespace

// Requests per transaction of the variable-length generator: uniform in
// [min_ops, max_ops], a pure function of (seed, tx).
static uint32_t var_ops(uint64_t seed, uint64_t tx, uint32_t lo, uint32_t hi) {
    return lo + (uint32_t)(hash3(seed ^ 0x4F505321ull, tx, 0) % (uint64_t)(hi - lo + 1));
}

extern "C" int gcc_gen_ycsb_var_offsets(uint64_t n_tx, uint32_t min_ops, uint32_t max_ops,
                                        uint64_t seed, uint32_t *tx_off) {
    if (!tx_off || min_ops < 1 || max_ops < min_ops || max_ops > 64) return GCC_EINVAL;
    uint64_t acc = 0;
    for (uint64_t t = 0; t < n_tx; ++t) {
        tx_off[t] = (uint32_t)acc;
        acc += var_ops(seed, t, min_ops, max_ops);
        if (acc > 0xFFFFFFFFull) return GCC_EINVAL;
    }
    tx_off[n_tx] = (uint32_t)acc;
    return GCC_OK;
}

extern "C" int gcc_gen_ycsb_var(uint64_t rows, uint64_t n_tx, double theta, double read_ratio,
                                uint64_t seed, int32_t key_base, int32_t threads,
                                const uint32_t *tx_off, gcc_ycsb_req *reqs) {
    if (!tx_off || (!reqs && n_tx)) return GCC_EINVAL;
    if (rows < 65 || rows > 0xFFFFFFFFull) return GCC_EINVAL;
    if (!(theta >= 0.0) || theta >= 1.0) return GCC_EINVAL;
    if (!(read_ratio >= 0.0) || read_ratio > 1.0) return GCC_EINVAL;
    if (key_base != 0 && key_base != 1) return GCC_EINVAL;
    for (uint64_t t = 0; t < n_tx; ++t)
        if (tx_off[t + 1] < tx_off[t] || tx_off[t + 1] - tx_off[t] > 64) return GCC_EINVAL;
    const uint64_t n = key_base == 1 ? rows - 1 : rows;
    const Zipf z(n, theta);
    unsigned nt = threads > 0 ? (unsigned)threads : std::max(1u, std::thread::hardware_concurrency());
    if ((uint64_t)nt > n_tx) nt = (unsigned)std::max<uint64_t>(1, n_tx);
    auto work = [&](uint64_t lo, uint64_t hi) {
        for (uint64_t t = lo; t < hi; ++t) {
            gcc_ycsb_req *rq = reqs + tx_off[t];
            const uint32_t want = tx_off[t + 1] - tx_off[t];
            uint64_t c = 0;
            uint32_t rid = 0;
            // distinct keys, redrawn on repeats (bounded), then key order
            for (uint32_t slot = 0; slot < want * 1024u && rid < want; ++slot) {
                double r = uniform(seed, t, c++);
                uint64_t rank = z.draw(uniform(seed, t, c++));
                uint32_t key = (uint32_t)(key_base == 1 ? rank : rank - 1);
                bool dup = false;
                for (uint32_t j = 0; j < rid; ++j) dup |= rq[j].key == key;
                if (dup) continue;
                rq[rid].read = r < read_ratio ? 1 : 0;
                rq[rid].key = key;
                ++rid;
            }
            // (practically unreachable for rows >= 65) take the smallest
            // unused keys so the transaction still has distinct keys
            for (uint32_t k = (uint32_t)key_base; rid < want; ++k) {
                bool used = false;
                for (uint32_t j = 0; j < rid; ++j) used |= rq[j].key == k;
                if (used) continue;
                rq[rid].read = 1;
                rq[rid].key = k;
                ++rid;
            }
            std::stable_sort(rq, rq + rid,
                             [](const gcc_ycsb_req &a, const gcc_ycsb_req &b) { return a.key < b.key; });
        }
    };
    std::vector<std::thread> pool;
    uint64_t per = (n_tx + nt - 1) / nt;
    for (unsigned i = 0; i < nt; ++i) {
        uint64_t lo = (uint64_t)i * per, hi = std::min<uint64_t>(n_tx, lo + per);
        if (lo >= hi) break;
        pool.emplace_back(work, lo, hi);
    }
    for (auto &th : pool) th.join();
    return GCC_OK;
}

extern "C" int gcc_gen_ycsb(uint64_t rows, uint64_t n_tx, double theta, double read_ratio,
                            uint64_t seed, int32_t dedup, int32_t key_base, int32_t threads,
                            gcc_ycsb_tx *out) {
    if (!out && n_tx) return GCC_EINVAL;
    if (rows < 3 || rows > 0xFFFFFFFFull) return GCC_EINVAL;
    if (!(theta >= 0.0) || theta >= 1.0) return GCC_EINVAL;  // theta = 1 divides by zero
    if (!(read_ratio >= 0.0) || read_ratio > 1.0) return GCC_EINVAL;
    if (dedup != GCC_DEDUP_DROP && dedup != GCC_DEDUP_RESAMPLE) return GCC_EINVAL;
    if (key_base != 0 && key_base != 1) return GCC_EINVAL;
    const uint64_t n = key_base == 1 ? rows - 1 : rows;
    const Zipf z(n, theta);
    unsigned nt = threads > 0 ? (unsigned)threads : std::max(1u, std::thread::hardware_concurrency());
    if ((uint64_t)nt > n_tx) nt = (unsigned)std::max<uint64_t>(1, n_tx);
    auto work = [&](uint64_t lo, uint64_t hi) {
        for (uint64_t t = lo; t < hi; ++t) {
            gcc_ycsb_tx &tx = out[t];
            memset(&tx, 0, sizeof(tx));
            uint64_t c = 0;
            int rid = 0;
            const int max_slots = dedup == GCC_DEDUP_DROP ? 16 : 16 * 1024;
            for (int slot = 0; slot < max_slots && rid < 16; ++slot) {
                double r = uniform(seed, t, c++);
                uint64_t rank = z.draw(uniform(seed, t, c++));
                uint32_t key = (uint32_t)(key_base == 1 ? rank : rank - 1);
                bool dup = false;
                for (int j = 0; j < rid; ++j) dup |= tx.requests[j].key == key;
                if (dup) continue;
                tx.requests[rid].read = r < read_ratio ? 1 : 0;
                tx.requests[rid].key = key;
                ++rid;
            }
            tx.request_cnt = (uint64_t)rid;
            std::stable_sort(tx.requests, tx.requests + rid,
                             [](const gcc_ycsb_req &a, const gcc_ycsb_req &b) { return a.key < b.key; });
        }
    };
    std::vector<std::thread> pool;
    uint64_t per = (n_tx + nt - 1) / nt;
    for (unsigned i = 0; i < nt; ++i) {
        uint64_t lo = (uint64_t)i * per, hi = std::min<uint64_t>(n_tx, lo + per);
        if (lo >= hi) break;
        pool.emplace_back(work, lo, hi);
    }
    for (auto &th : pool) th.join();
    return GCC_OK;
}
