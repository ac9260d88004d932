"""The predictor's CPU oracle checked against itself by independent means:
its analytic gradient against central finite differences of its loss, its
BF16 rounding against known bit patterns, and its features against a direct
per-request count. These pin the checker that the GPU predictor is compared
with in test_gpu_sched.py."""
import numpy as np

import gpu_cc_tb_b200 as g
from oracle import predictor as P


def _rand_feat(rng, n):
    f = np.zeros((n, P.FEAT_STRIDE), dtype=np.uint16)
    f[:, :64] = rng.integers(0, 3, size=(n, 64))
    f[:, 64] = rng.integers(0, 17, size=n)
    f[:, 65] = rng.integers(0, 17, size=n)
    return f


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    w = rng.normal(0, 0.15, P.N_PARAMS)
    feat = _rand_feat(rng, 64)
    y = rng.integers(0, 2, 64).astype(np.uint8)
    loss, grad = P.loss_and_grad(w, feat, y, bf16=False)
    idx = np.concatenate([rng.choice(np.arange(P.OFF_W1, P.OFF_B1), 12, replace=False),
                          rng.choice(np.arange(P.OFF_B1, P.OFF_W2), 4, replace=False),
                          rng.choice(np.arange(P.OFF_W2, P.OFF_B2), 12, replace=False),
                          rng.choice(np.arange(P.OFF_B2, P.OFF_W3), 4, replace=False),
                          rng.choice(np.arange(P.OFF_W3, P.OFF_B3), 6, replace=False), [P.OFF_B3]])
    h = 1e-6
    for i in idx:
        wp, wm = w.copy(), w.copy()
        wp[i] += h
        wm[i] -= h
        fd = (P.loss_and_grad(wp, feat, y, bf16=False)[0] -
              P.loss_and_grad(wm, feat, y, bf16=False)[0]) / (2 * h)
        assert abs(fd - grad[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, grad[i])
    assert np.isfinite(loss) and loss > 0


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -2.5, 3.0e-3, 65504.0], dtype=np.float32)
    r = P.bf16_round(x)
    bits = r.view(np.uint32)
    assert (bits & 0xFFFF).max() == 0
    assert r[0] == 1.0
    assert r[1] == 1.0                 # halfway (1 + 2^-8), ties to even
    assert r[2] == np.float32(1.0078125)  # above halfway rounds up
    assert r[3] == -2.5


def test_features_direct_count():
    rows = 5000
    txs = g.gen_ycsb(rows, 300, 0.9, 0.7, seed=5, dedup=g.DEDUP_DROP, key_base=0)
    freq = np.zeros(1 << P.FREQ_BITS, dtype=np.uint32)
    for _ in range(3):
        freq = P.observe(freq, txs)
    f = P.features(txs, freq)
    for t in range(0, 300, 37):
        n = int(txs[t]["request_cnt"])
        keys = txs[t]["requests"]["key"][:n].astype(np.uint64)
        reads = txs[t]["requests"]["read"][:n]
        sk = np.zeros(64, dtype=np.int64)
        for k in keys:
            sk[int(P.splitmix64(np.array([k]))[0] & np.uint64(63))] += 1
        assert np.array_equal(f[t, :64], sk)
        assert f[t, 64] == int((reads == 0).sum())
        # floor(log2(1 + c)) per request, by integer bit length
        heat = sum((int(freq[P.freq_slots(np.array([k]))[0]]) + 1).bit_length() - 1 for k in keys)
        assert f[t, 65] == heat
        assert not f[t, 66:].any()


def test_lock_plan_known_answer():
    # one record: keys 3, 9, 20, 40, 50 (request order); counters chosen so
    # that keys 9 and 40 tie, key 50 is the hottest and key 3 is cold
    txs = np.zeros(1, dtype=g.TX_DTYPE)
    keys = [3, 9, 20, 40, 50]
    txs[0]["request_cnt"] = len(keys)
    for i, k in enumerate(keys):
        txs[0]["requests"][i] = (1 if i % 2 else 0, k)
    freq = np.zeros(1 << P.FREQ_BITS, dtype=np.uint32)
    cnt = {3: 5, 9: 300, 20: 1000, 40: 300, 50: 7000}
    slots = P.freq_slots(np.array(keys, dtype=np.uint64))
    assert len(set(slots.tolist())) == len(keys)
    for k, sl in zip(keys, slots):
        freq[sl] = cnt[k]
    plan = int(P.lock_plans(txs, freq, 100)[0])
    # planned: requests 1 (key 9), 3 (key 40), 2 (key 20), 4 (key 50), in
    # that order: (300, 9) < (300, 40) < (1000, 20) < (7000, 50)
    assert plan & 0xFFFF == 0b11110
    assert (plan >> 16) & 0xF == 4
    assert [(plan >> (20 + 4 * j)) & 0xF for j in range(4)] == [1, 3, 2, 4]
    # a threshold above every counter plans nothing
    assert int(P.lock_plans(txs, freq, 10_000)[0]) == 0
    # more than 11 hot requests: only the 11 hottest are planned
    txs2 = np.zeros(1, dtype=g.TX_DTYPE)
    txs2[0]["request_cnt"] = 16
    keys2 = np.arange(100, 116, dtype=np.uint64)
    for i in range(16):
        txs2[0]["requests"][i] = (1, int(keys2[i]))
    freq2 = np.zeros(1 << P.FREQ_BITS, dtype=np.uint32)
    for i, sl in enumerate(P.freq_slots(keys2)):
        freq2[sl] = max(freq2[sl], 1000 + i)
    plan2 = int(P.lock_plans(txs2, freq2, 1)[0])
    assert (plan2 >> 16) & 0xF == 11
    order = [(plan2 >> (20 + 4 * j)) & 0xF for j in range(11)]
    assert order == sorted(order) and order[-1] == 15
