"""ctypes loader of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE: imported only by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, always as the checker or the timed CPU
baseline, never as part of the engine.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
_lib = None


def build():
    src = [HERE / "oracle.cpp", HERE / "oracle.h"]
    if not LIB.exists() or LIB.stat().st_mtime < max(p.stat().st_mtime for p in src):
        subprocess.run(["make", "-C", str(HERE), "-s"], check=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(str(LIB))
        P, U64, I32 = C.c_void_p, C.c_uint64, C.c_int32
        sig = {
            "oracle_fill_table": [U64, I32, U64, P],
            "oracle_replay": [P, U64, I32, P, U64, P, U64, I32, U64, P, P],
            "oracle_gputx_order": [P, U64, U64, P, P, P],
            "oracle_replay_var": [P, U64, I32, P, P, U64, P, U64, I32, U64, P],
            "oracle_replay_var_ext": [P, U64, I32, P, P, U64, P, U64, I32, U64, P, I32],
            "oracle_commit_order": [P, U64, P],
            "oracle_conflict_acyclic": [P, U64, U64],
            "oracle_cpu_run": [C.c_char_p, P, U64, I32, P, U64, I32, U64, I32, P, P,
                               C.POINTER(C.c_double), C.POINTER(U64)],
            "oracle_gen_ycsb": [U64, U64, C.c_double, C.c_double, U64, I32, I32, P],
            "oracle_cpu_run_var": [C.c_char_p, P, U64, I32, P, P, U64, I32, U64, I32, I32, P, P,
                                   C.POINTER(C.c_double), C.POINTER(U64)],
        }
        for name, args in sig.items():
            fn = getattr(L, name)
            fn.restype = C.c_int
            fn.argtypes = args
        _lib = L
    return _lib


def _p(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


def rbytes(layout):
    return 104 if layout == 1 else 88


def rstride(layout):
    return 112 if layout == 1 else 96


def fill_table(rows, layout, seed):
    t = np.empty((rows, rbytes(layout)), dtype=np.uint8)
    rc = lib().oracle_fill_table(rows, layout, seed, _p(t))
    assert rc == 0, rc
    return t


def replay(table, layout, txs, order, write_mode, write_seed, read_log=False):
    """Serially execute txs[order] over a copy of `table`; returns
    (final_table, digests[n_tx], read_log or None). Txs not in `order` keep
    digest 0."""
    t = np.array(table, dtype=np.uint8, copy=True)
    n = len(txs)
    dg = np.zeros(n, dtype=np.uint64)
    order = np.ascontiguousarray(np.arange(n) if order is None else order, dtype=np.uint32)
    rl = np.zeros((n, 16, rstride(layout)), dtype=np.uint8) if read_log else None
    rc = lib().oracle_replay(_p(t), t.shape[0], layout, _p(txs), n, _p(order), len(order),
                             write_mode, write_seed, _p(dg), _p(rl))
    if rc != 0:
        raise RuntimeError(f"oracle_replay failed: {rc}")
    return t, dg, rl


def replay_var(table, layout, tx_off, reqs, order, write_mode, write_seed, ext_ops=False):
    """Serial replay of variable-length transactions (CSR); ext_ops applies
    extended request ops (negative `read` words)."""
    t = np.array(table, dtype=np.uint8, copy=True)
    n = len(tx_off) - 1
    dg = np.zeros(n, dtype=np.uint64)
    order = np.ascontiguousarray(np.arange(n) if order is None else order, dtype=np.uint32)
    tx_off = np.ascontiguousarray(tx_off, dtype=np.uint32)
    reqs = np.ascontiguousarray(reqs)
    rc = lib().oracle_replay_var_ext(_p(t), t.shape[0], layout, _p(tx_off), _p(reqs), n, _p(order),
                                     len(order), write_mode, write_seed, _p(dg), 1 if ext_ops else 0)
    if rc != 0:
        raise RuntimeError(f"oracle_replay_var failed: {rc}")
    return t, dg


def gputx_order(txs, rows):
    n = len(txs)
    ranks = np.zeros(n, dtype=np.uint32)
    order = np.zeros(n, dtype=np.uint32)
    mx = np.zeros(1, dtype=np.uint32)
    rc = lib().oracle_gputx_order(_p(txs), n, rows, _p(ranks), _p(order), _p(mx))
    assert rc == 0, rc
    return ranks, order, int(mx[0])


def commit_order(log):
    log = np.ascontiguousarray(log, dtype=np.uint64)
    order = np.zeros(len(log), dtype=np.uint32)
    rc = lib().oracle_commit_order(_p(log), len(log), _p(order))
    assert rc == 0
    return order


EVENT_DTYPE = np.dtype([("tx", "<u4"), ("row", "<u4"), ("is_write", "<u4"), ("pad", "<u4"),
                        ("seq", "<u8")])


def conflict_acyclic(events, n_tx):
    ev = np.ascontiguousarray(events, dtype=EVENT_DTYPE)
    return bool(lib().oracle_conflict_acyclic(_p(ev), len(ev), n_tx))


def cpu_run(scheme, table, layout, txs, write_mode, write_seed, threads=0, commit_log=True):
    t = np.array(table, dtype=np.uint8, copy=True)
    n = len(txs)
    dg = np.zeros(n, dtype=np.uint64)
    log = np.zeros((n, 2), dtype=np.uint64) if commit_log else None
    secs, aborts = C.c_double(), C.c_uint64()
    rc = lib().oracle_cpu_run(scheme.encode(), _p(t), t.shape[0], layout, _p(txs), n, write_mode,
                              write_seed, threads, _p(dg), _p(log), C.byref(secs),
                              C.byref(aborts))
    if rc != 0:
        raise RuntimeError(f"oracle_cpu_run failed: {rc}")
    return t, dg, log, secs.value, aborts.value


def cpu_run_var(scheme, table, layout, tx_off, reqs, write_mode, write_seed, ext_ops=False,
                threads=0, commit_log=True):
    """Multi-threaded CPU execution of variable-length transactions."""
    t = np.array(table, dtype=np.uint8, copy=True)
    tx_off = np.ascontiguousarray(tx_off, dtype=np.uint32)
    reqs = np.ascontiguousarray(reqs)
    n = len(tx_off) - 1
    dg = np.zeros(n, dtype=np.uint64)
    log = np.zeros((n, 2), dtype=np.uint64) if commit_log else None
    secs, aborts = C.c_double(), C.c_uint64()
    rc = lib().oracle_cpu_run_var(scheme.encode(), _p(t), t.shape[0], layout, _p(tx_off), _p(reqs),
                                  n, write_mode, write_seed, 1 if ext_ops else 0, threads, _p(dg),
                                  _p(log), C.byref(secs), C.byref(aborts))
    if rc != 0:
        raise RuntimeError(f"oracle_cpu_run_var failed: {rc}")
    return t, dg, log, secs.value, aborts.value


# gen_ycsb record: {uint64 request_cnt; {int32 read; uint32 key}[16]} = 136 B
# (include/ycsb.cuh:21-33 of the reference)
TX_DTYPE = np.dtype([("request_cnt", "<u8"),
                     ("requests", np.dtype([("read", "<i4"), ("key", "<u4")]), (16,))])


def gen_ycsb(rows, n_tx, theta, read_ratio, seed, dedup, key_base):
    """The oracle's restatement of the dataset generator (same records as
    the engine's gcc_gen_ycsb for the same arguments)."""
    out = np.zeros(n_tx, dtype=TX_DTYPE)
    rc = lib().oracle_gen_ycsb(rows, n_tx, theta, read_ratio, seed, dedup, key_base, _p(out))
    assert rc == 0, rc
    return out


_M64 = (1 << 64) - 1


def _sm64(x):
    z = (x + 0x9E3779B97F4A7C15) & _M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M64
    return z ^ (z >> 31)


def _h3(s, a, b):
    return _sm64(_sm64(s ^ ((a * 0x9E3779B97F4A7C15) & _M64)) ^ ((b * 0xC2B2AE3D27D4EB4F) & _M64))


def write_field(write_seed, tx, op):
    """Field (0..9) a GCC_WRITE_FIELD write request `op` of transaction `tx`
    stores into (the formula oracle.cpp's replay applies)."""
    return _h3(write_seed, tx, 2 * op) % 10


def write_value(write_seed, tx, op):
    """Value that write request `op` of transaction `tx` stores."""
    return _h3(write_seed, tx, 2 * op + 1)


def gputx_rank_hazards(txs, rows):
    """Where the reference's GPUTx run is not deterministic on `txs`, so
    that its output cannot be compared byte for byte: (same_rank_conflicts,
    last_object_accesses).
      same_rank_conflicts: (row, rank) groups that two or more transactions
        of the same rank access with at least one write; the reference runs
        a rank in one launch without ordering them (src/gputx.cu:17-27,
        include/gputx.cuh:289-294);
      last_object_accesses: accesses to the highest accessed row; the
        reference's rank pass reads that row's list end one past its scanned
        offsets (offset[dense_cnt], include/gputx.cuh:252-253 and
        src/gputx.cu:17-18), so only a row accessed once ranks the same."""
    ranks, _, _ = gputx_order(txs, rows)
    cnt = txs["request_cnt"].astype(np.int64)
    valid = np.arange(16)[None, :] < cnt[:, None]
    t = np.broadcast_to(np.arange(len(txs))[:, None], valid.shape)[valid]
    k = txs["requests"]["key"].astype(np.int64)[valid]
    w = (txs["requests"]["read"] == 0)[valid]
    r = np.asarray(ranks, dtype=np.int64)[t]
    o = np.lexsort((t, r, k))
    k, r, w = k[o], r[o], w[o]
    start = np.ones(len(k), dtype=bool)
    start[1:] = (k[1:] != k[:-1]) | (r[1:] != r[:-1])
    gid = np.cumsum(start) - 1
    size = np.bincount(gid)
    anyw = np.bincount(gid, weights=w.astype(np.float64)) > 0
    same_rank = int(((size >= 2) & anyw).sum())
    last = int((k == k.max()).sum()) if len(k) else 0
    return same_rank, last
