"""CPU oracle of the learned contention predictor (features, frequency table,
network, loss and gradient), in numpy and float64.

TEST INFRASTRUCTURE: imported only by tests/ (as the checker of the CUDA
predictor), never by the engine.

It restates, independently of gpu_cc_tb_b200/csrc/sched.cu, the definitions
the engine's predictor implements:
  * features of a transaction (66 values): a 64-bin count sketch of its keys
    (bin = splitmix64(key) & 63), its number of write requests, and the sum
    over its requests of floor(log2(1 + c)), c the key's counter in the
    frequency table;
    the table has 2^20 counters indexed by splitmix64(key ^ 0x5EEDF00D) >> 44
    and after each batch is halved, then incremented once per request;
  * the network 66 -> 128 -> 128 -> 1 on features / 16, ReLU hidden layers,
    sigmoid output, with weights rounded to BF16 (round to nearest even);
  * the mean binary cross-entropy against 0/1 labels and its gradient with
    respect to every parameter (flat layout W1[66][128], b1, W2[128][128],
    b2, w3[128], b3);
  * the 2PL lock plan of a transaction: which requests are locked after the
    others (key counter >= a threshold) and in which order (the hottest
    last).
The predictor has no counterpart in the reference (gCCTB runs transactions
in index order); these definitions are the checker for the GPU kernels, and
the gradient itself is pinned by finite differences in tests/.
"""
from __future__ import annotations

import numpy as np

N_IN, N_HID, FEAT_STRIDE, FREQ_BITS = 66, 128, 72, 20
OFF_W1 = 0
OFF_B1 = OFF_W1 + N_IN * N_HID
OFF_W2 = OFF_B1 + N_HID
OFF_B2 = OFF_W2 + N_HID * N_HID
OFF_W3 = OFF_B2 + N_HID
OFF_B3 = OFF_W3 + N_HID
N_PARAMS = OFF_B3 + 1

def splitmix64(x: np.ndarray) -> np.ndarray:
    x = np.asarray(x, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = x + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def _keys(txs):
    keys = txs["requests"]["key"].astype(np.uint64)
    reads = txs["requests"]["read"]
    mask = np.arange(16)[None, :] < txs["request_cnt"].astype(np.int64)[:, None]
    return keys, reads, mask


def freq_slots(keys: np.ndarray) -> np.ndarray:
    return (splitmix64(keys ^ np.uint64(0x5EEDF00D)) >> np.uint64(64 - FREQ_BITS)).astype(np.int64)


def observe(freq: np.ndarray, txs) -> np.ndarray:
    """Frequency table after one batch: halve, then count every request."""
    keys, _, mask = _keys(txs)
    f = freq >> np.uint32(1)
    np.add.at(f, freq_slots(keys)[mask], np.uint32(1))
    return f


def features(txs, freq: np.ndarray) -> np.ndarray:
    """u16 feature rows of stride 72 (columns 66..71 zero)."""
    keys, reads, mask = _keys(txs)
    n = len(txs)
    out = np.zeros((n, FEAT_STRIDE), dtype=np.uint16)
    bins = (splitmix64(keys) & np.uint64(63)).astype(np.int64)
    rows = np.repeat(np.arange(n), 16).reshape(n, 16)
    np.add.at(out, (rows[mask], bins[mask]), 1)
    out[:, 64] = (mask & (reads == 0)).sum(axis=1)
    c = freq[freq_slots(keys)].astype(np.uint64) + np.uint64(1)
    heat = np.floor(np.log2(c.astype(np.float64))).astype(np.int64)
    out[:, 65] = (np.where(mask, heat, 0)).sum(axis=1)
    return out


def bf16_round(w: np.ndarray) -> np.ndarray:
    u = np.ascontiguousarray(w, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = (u + np.uint64(0x7FFF) + ((u >> np.uint64(16)) & np.uint64(1))) & np.uint64(0xFFFF0000)
    return r.astype(np.uint32).view(np.float32)


def unpack(w: np.ndarray, bf16: bool = True):
    w = bf16_round(w).astype(np.float64) if bf16 else np.asarray(w, dtype=np.float64)
    W1 = w[OFF_W1:OFF_B1].reshape(N_IN, N_HID)
    b1 = w[OFF_B1:OFF_W2]
    W2 = w[OFF_W2:OFF_B2].reshape(N_HID, N_HID)
    b2 = w[OFF_B2:OFF_W3]
    w3 = w[OFF_W3:OFF_B3]
    b3 = w[OFF_B3]
    return W1, b1, W2, b2, w3, b3


def forward(w: np.ndarray, feat: np.ndarray, bf16: bool = True):
    W1, b1, W2, b2, w3, b3 = unpack(w, bf16)
    x = feat[:, :N_IN].astype(np.float64) / 16.0
    h1 = np.maximum(x @ W1 + b1, 0.0)
    h2 = np.maximum(h1 @ W2 + b2, 0.0)
    z = h2 @ w3 + b3
    p = 1.0 / (1.0 + np.exp(-z))
    return x, h1, h2, z, p


def loss_and_grad(w: np.ndarray, feat: np.ndarray, y: np.ndarray, bf16: bool = True):
    """(mean BCE, gradient[N_PARAMS]) at the BF16-rounded weights (at the
    weights as given with bf16=False)."""
    W1, b1, W2, b2, w3, b3 = unpack(w, bf16)
    x, h1, h2, z, p = forward(w, feat, bf16)
    y = np.asarray(y, dtype=np.float64)
    n = len(y)
    loss = float(np.mean(np.maximum(z, 0) + np.log1p(np.exp(-np.abs(z))) - y * z))
    dz = (p - y) / n
    g = np.zeros(N_PARAMS, dtype=np.float64)
    g[OFF_W3:OFF_B3] = h2.T @ dz
    g[OFF_B3] = dz.sum()
    dh2 = np.outer(dz, w3) * (h2 > 0)
    g[OFF_W2:OFF_B2] = (h1.T @ dh2).ravel()
    g[OFF_B2:OFF_W3] = dh2.sum(axis=0)
    dh1 = (dh2 @ W2.T) * (h1 > 0)
    g[OFF_W1:OFF_B1] = (x.T @ dh1).ravel()
    g[OFF_B1:OFF_W2] = dh1.sum(axis=0)
    return loss, g


def _var_keys(tx_off, reqs, lo, hi):
    """Per-request (tx index, key, read word) of transactions lo .. hi-1."""
    a, b = int(tx_off[lo]), int(tx_off[hi])
    cnt = np.diff(tx_off[lo:hi + 1]).astype(np.int64)
    tx = np.repeat(np.arange(hi - lo), cnt)
    return tx, reqs["key"][a:b].astype(np.uint64), reqs["read"][a:b]


PLAN_MAX = 11


def lock_plans(txs, freq: np.ndarray, thr: int) -> np.ndarray:
    """2PL lock plan of each record (the scheduler's k_lock_plan): requests
    whose key counter c >= thr, ordered by (c, key) ascending; at most
    PLAN_MAX of them, the last ones of that order. u64: bits 0-15 the planned
    requests, 16-19 their count, nibble j at bit 20 + 4j the j-th request
    index. Pure-Python loop over records (small cases)."""
    keys, _, mask = _keys(txs)
    c = freq[freq_slots(keys)].astype(np.int64)
    out = np.zeros(len(txs), dtype=np.uint64)
    for t in range(len(txs)):
        hot = [(int(c[t, i]), int(keys[t, i]), i) for i in range(16)
               if mask[t, i] and c[t, i] >= thr]
        hot.sort()
        hot = hot[max(0, len(hot) - PLAN_MAX):]
        v = len(hot) << 16
        for j, (_, _, i) in enumerate(hot):
            v |= (1 << i) | (i << (20 + 4 * j))
        out[t] = v
    return out


def observe_var(freq: np.ndarray, tx_off, reqs, lo, hi) -> np.ndarray:
    """observe() for variable-length transactions lo .. hi-1 (CSR)."""
    _, keys, _ = _var_keys(tx_off, reqs, lo, hi)
    f = freq >> np.uint32(1)
    np.add.at(f, freq_slots(keys), np.uint32(1))
    return f


def features_var(tx_off, reqs, lo, hi, freq: np.ndarray) -> np.ndarray:
    """features() for variable-length transactions lo .. hi-1: every request
    counts (writes are requests whose read word is <= 0)."""
    tx, keys, reads = _var_keys(tx_off, reqs, lo, hi)
    out = np.zeros((hi - lo, FEAT_STRIDE), dtype=np.uint16)
    bins = (splitmix64(keys) & np.uint64(63)).astype(np.int64)
    np.add.at(out, (tx, bins), 1)
    np.add.at(out[:, 64], tx, (reads <= 0).astype(np.uint16))
    c = freq[freq_slots(keys)].astype(np.uint64) + np.uint64(1)
    heat = np.floor(np.log2(c.astype(np.float64))).astype(np.uint16)
    np.add.at(out[:, 65], tx, heat)
    return out
