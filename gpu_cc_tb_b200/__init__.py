"""B200 transaction-execution engine for gCCTB's YCSB hot path.

Python mirror of the C ABI in ``include/gcc_engine.h`` (ctypes over the
in-tree ``lib/libgcctb.so``). It exposes the reference's operator surface:
the ``cc_scheme`` names, the ``warp_density`` / ``block_size`` /
``batch_size`` knobs, the gen_ycsb dataset records (136-byte ``YCSBTx``) and
the 15-column result line of ``test_ycsb`` (gCCTB
``benchmark_cpu/ycsb.cu:81-302``, ``include/runtime.cuh:169-214``).

There is no CPU execution path: every run goes through the CUDA library, and
importing fails loudly when it is missing.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

__all__ = [
    "SCHEMES", "LAYOUT_U64X11", "LAYOUT_REF104", "INDEX_HASH", "INDEX_SORTED",
    "INDEX_DIRECT", "WRITE_FIELD", "WRITE_ROWCOPY", "F_COMMIT_LOG", "F_READ_LOG",
    "F_NO_RESET", "DEDUP_DROP", "DEDUP_RESAMPLE", "TX_DTYPE", "GccError", "Engine",
    "gen_ycsb", "library", "library_path", "scheme_id", "row_bytes", "row_stride",
    "gen_ycsb_var", "REQ_DTYPE", "F_RETRY_IMMEDIATE", "F_AUTOTUNE", "F_GRAPH",
    "BATCHES_SEQUENTIAL", "BATCHES_QUEUE", "VAR_SCHEMES",
]

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "lib" / "libgcctb.so"

# cc_scheme names of test_ycsb (benchmark_cpu/ycsb.cu:168-195)
SCHEMES = ("tpl_nw", "tpl_wd", "to", "mvcc", "silo", "tictoc", "gacco", "gputx",
           "slow_tpl_nw", "slow_tpl_wd", "slow_to", "slow_mvcc", "slow_silo", "slow_tictoc")

LAYOUT_U64X11, LAYOUT_REF104 = 0, 1
INDEX_HASH, INDEX_SORTED, INDEX_DIRECT = 0, 1, 2
WRITE_FIELD, WRITE_ROWCOPY = 0, 1
F_COMMIT_LOG, F_READ_LOG, F_NO_RESET, F_RETRY_IMMEDIATE = 1, 2, 4, 8
F_AUTOTUNE, F_GRAPH = 16, 32
F_QUEUE = 128  # gcc_run / gcc_run_host: all batches through one device-queue launch
F_REQUEST_ORDER = 256  # 2PL / TO one-at-a-time retries in request order (the reference's)
QUEUE_SCHEMES = ("tpl_nw", "tpl_wd", "to", "silo", "tictoc", "slow_tpl_nw", "slow_tpl_wd",
                 "slow_to", "slow_silo", "slow_tictoc")
BATCHES_SEQUENTIAL, BATCHES_QUEUE = 0, 1
DEDUP_DROP, DEDUP_RESAMPLE = 0, 1

STATUS = {0: "GCC_OK", -1: "GCC_EINVAL", -2: "GCC_ENOMEM", -3: "GCC_ECUDA", -4: "GCC_ETIMEOUT",
          -5: "GCC_EFORMAT", -6: "GCC_EKEY", -7: "GCC_EOVERFLOW", -8: "GCC_ESTATE",
          -9: "GCC_ENODEV"}

# gen_ycsb record: {size_t request_cnt; {int read; unsigned key;}[16]} = 136 B
TX_DTYPE = np.dtype([("request_cnt", "<u8"),
                     ("requests", np.dtype([("read", "<i4"), ("key", "<u4")]), (16,))])
assert TX_DTYPE.itemsize == 136
REQ_DTYPE = np.dtype([("read", "<i4"), ("key", "<u4")])
# schemes of the batched executors (gcc_run_batches); mvcc: sequential only
VAR_SCHEMES = ("tpl_nw", "tpl_wd", "to", "silo", "tictoc", "mvcc", "slow_tpl_nw", "slow_tpl_wd",
               "slow_to", "slow_silo", "slow_tictoc", "slow_mvcc")


class GccError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        name = STATUS.get(status, str(status))
        msg = library().gcc_strerror(status).decode()
        super().__init__(f"{what}: {name} ({msg})" if what else f"{name} ({msg})")


class TableDesc(C.Structure):
    _fields_ = [("rows", C.c_uint64), ("layout", C.c_int32), ("index_kind", C.c_int32),
                ("fill_seed", C.c_uint64), ("device", C.c_int32), ("max_batch", C.c_int32)]


class RunParams(C.Structure):
    _fields_ = [("cc_scheme", C.c_char_p), ("warp_density", C.c_int32),
                ("block_size", C.c_int32), ("batch_size", C.c_int32), ("flags", C.c_uint32),
                ("write_mode", C.c_int32), ("backoff_ns", C.c_int32), ("write_seed", C.c_uint64),
                ("spin_limit_ns", C.c_uint64),
                ("starve_limit", C.c_int32), ("max_active", C.c_int32),
                ("ordered_after", C.c_int32), ("reserved", C.c_int32)]


class Result(C.Structure):
    _fields_ = [("tx_per_s", C.c_double), ("committed", C.c_uint64), ("aborts", C.c_uint64),
                ("ts_d", C.c_double), ("wait_d", C.c_double), ("abort_d", C.c_double),
                ("mng_d", C.c_double), ("tot_d", C.c_double), ("idx_d", C.c_double),
                ("pre_s", C.c_double), ("proc_s", C.c_double), ("tot_s", C.c_double),
                ("lat_p50_us", C.c_double), ("lat_p99_us", C.c_double),
                ("rank_count", C.c_uint64), ("batches", C.c_uint64),
                ("kernel_launches", C.c_uint64), ("max_attempts", C.c_uint32),
                ("err_site", C.c_uint32)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class CommitRec(C.Structure):
    _fields_ = [("hi", C.c_uint64), ("lo", C.c_uint64)]


_LIB = None


class SchedParams(C.Structure):
    _fields_ = [("mode", C.c_int32), ("explore_every", C.c_int32), ("probe_rows", C.c_int32),
                ("train_steps", C.c_int32), ("minibatch", C.c_int32), ("lr", C.c_float),
                ("defer_threshold", C.c_float), ("fixed_arm", C.c_int32), ("min_sched", C.c_int32),
                ("plan_threshold", C.c_int32), ("seed", C.c_uint64), ("plan_after", C.c_int32),
                ("reserved", C.c_int32)]


class SchedBatch(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("bucket", C.c_uint32), ("arm", C.c_uint32),
                ("in_flight_cap", C.c_uint32), ("wait_die", C.c_uint32), ("probe", C.c_uint32),
                ("deferred", C.c_uint64), ("pred_mean", C.c_float), ("label_mean", C.c_float),
                ("loss", C.c_float), ("explored", C.c_uint32), ("ms", C.c_double),
                ("committed", C.c_uint64), ("aborts", C.c_uint64)]


class SchedResult(C.Structure):
    _fields_ = [("run", Result), ("probed", C.c_uint64), ("deferred", C.c_uint64),
                ("probe_tx_per_s", C.c_double), ("sched_tx_per_s", C.c_double),
                ("probe_abort_rate", C.c_double), ("sched_abort_rate", C.c_double),
                ("predict_ms", C.c_double), ("train_ms", C.c_double), ("last_loss", C.c_double)]


class OeDesc(C.Structure):
    _fields_ = [("warehouses", C.c_uint32), ("districts", C.c_uint32), ("customers", C.c_uint32),
                ("items", C.c_uint32), ("new_order_pct", C.c_uint32),
                ("remote_line_permille", C.c_uint32), ("remote_customer_pct", C.c_uint32),
                ("min_lines", C.c_uint32), ("max_lines", C.c_uint32)]


class OeLayout(C.Structure):
    _fields_ = [("warehouse", C.c_uint64), ("district", C.c_uint64), ("customer", C.c_uint64),
                ("item", C.c_uint64), ("stock", C.c_uint64), ("inserts", C.c_uint64),
                ("rows", C.c_uint64)]


OP_ADD, OP_SUB, OP_STOCK, OP_PAY, OP_INSERT = 1, 2, 3, 4, 5
F_EXT_OPS = 64


def op_word(op: int, field: int, v: int) -> int:
    """The `read` word of an extended request op (GCC_OP_WORD)."""
    return int(np.int32(np.uint32(0x80000000 | (op << 28) | (field << 24) | (v & 0xFFFFFF)).view(np.int32)))


class ServeParams(C.Structure):
    _fields_ = [("rate_tps", C.c_double), ("seed", C.c_uint64), ("max_batch", C.c_int32),
                ("min_batch", C.c_int32), ("max_wait_us", C.c_double)]


class ServeResult(C.Structure):
    _fields_ = [("committed", C.c_uint64), ("aborts", C.c_uint64), ("batches", C.c_uint64),
                ("admit_cap", C.c_uint64), ("offered_tps", C.c_double), ("tx_per_s", C.c_double),
                ("device_tx_per_s", C.c_double), ("lat_p50_us", C.c_double),
                ("lat_p99_us", C.c_double), ("lat_max_us", C.c_double), ("mean_batch", C.c_double),
                ("busy_frac", C.c_double), ("sched_abort_rate", C.c_double),
                ("kernel_launches", C.c_uint64)]


SCHED_PLAIN, SCHED_LEARNED = 0, 1
SCHED_FEAT_STRIDE = 72
SCHED_SCHEMES = ["tpl_nw", "tpl_wd", "silo", "tictoc"]


CALIB_ADD, CALIB_CAS = 0, 1


def l2_atomic_rate(device: int = 0, words: int = 1 << 23, mode: int = CALIB_ADD) -> float:
    """64-bit L2 atomics per second the device sustains on pseudo-random words
    of a `words`-word array (gcc_l2_atomic_rate)."""
    r = C.c_double()
    _check(library().gcc_l2_atomic_rate(device, words, mode, C.byref(r)), "gcc_l2_atomic_rate")
    return r.value


def library_path() -> Path:
    return Path(os.environ.get("GCC_LIB", LIB_PATH))


def library() -> C.CDLL:
    """Load the CUDA C-ABI library (built by gpu_cc_tb_b200/build.py)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = library_path()
    if not path.exists():
        raise ImportError(f"{path} is missing: build it with `python gpu_cc_tb_b200/build.py`")
    lib = C.CDLL(str(path))
    P = C.c_void_p
    sig = {
        "gcc_version": (C.c_char_p, []),
        "gcc_strerror": (C.c_char_p, [C.c_int]),
        "gcc_scheme_id": (C.c_int, [C.c_char_p]),
        "gcc_row_bytes": (C.c_uint32, [C.c_int32]),
        "gcc_row_stride": (C.c_uint32, [C.c_int32]),
        "gcc_gen_ycsb": (C.c_int, [C.c_uint64, C.c_uint64, C.c_double, C.c_double, C.c_uint64,
                                   C.c_int32, C.c_int32, C.c_int32, P]),
        "gcc_create": (C.c_int, [C.POINTER(TableDesc), C.POINTER(P)]),
        "gcc_destroy": (None, [P]),
        "gcc_load_txs": (C.c_int, [P, P, C.c_uint64]),
        "gcc_run": (C.c_int, [P, C.POINTER(RunParams), C.POINTER(Result)]),
        "gcc_run_host": (C.c_int, [P, C.POINTER(RunParams), P, C.c_uint64, P, C.POINTER(Result)]),
        "gcc_run_checked": (C.c_int, [P, C.POINTER(RunParams), C.POINTER(Result),
                                      C.POINTER(C.c_int)]),
        "gcc_format_line": (C.c_int, [C.POINTER(RunParams), C.POINTER(Result), C.c_char_p,
                                      C.c_size_t]),
        "gcc_dump_table": (C.c_int, [P, P, C.c_uint64]),
        "gcc_upload_table": (C.c_int, [P, P, C.c_uint64]),
        "gcc_get_digests": (C.c_int, [P, P, C.c_uint64]),
        "gcc_get_commit_log": (C.c_int, [P, P, C.c_uint64]),
        "gcc_get_tx_aborts": (C.c_int, [P, P, C.c_uint64]),
        "gcc_get_read_log": (C.c_int, [P, P, C.c_uint64]),
        "gcc_index_lookup": (C.c_int, [P, P, P, C.c_uint64]),
        "gcc_last_kernel_ms": (C.c_int, [P, C.POINTER(C.c_double), C.POINTER(C.c_uint64)]),
        "gcc_l2_atomic_rate": (C.c_int, [C.c_int32, C.c_uint64, C.c_int32,
                                         C.POINTER(C.c_double)]),
        "gcc_gen_ycsb_var_offsets": (C.c_int, [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint64, P]),
        "gcc_gen_ycsb_var": (C.c_int, [C.c_uint64, C.c_uint64, C.c_double, C.c_double,
                                       C.c_uint64, C.c_int32, C.c_int32, P, P]),
        "gcc_load_var_txs": (C.c_int, [P, P, P, C.c_uint64]),
        "gcc_run_batches": (C.c_int, [P, C.POINTER(RunParams), P, C.c_uint64, C.c_int32,
                                      C.POINTER(Result)]),
        "gcc_get_batch_stats": (C.c_int, [P, P, P, P, C.c_uint64]),
        "gcc_get_batch_active": (C.c_int, [P, P, C.c_uint64]),
        "gcc_get_batch_split": (C.c_int, [P, P, C.c_uint64]),
        "gcc_oe_offsets": (C.c_int, [C.POINTER(OeDesc), C.c_uint64, C.c_uint64, P,
                                     C.POINTER(OeLayout)]),
        "gcc_oe_gen": (C.c_int, [C.POINTER(OeDesc), C.c_uint64, C.c_uint64, C.c_int32, P, P, P]),
        "gcc_oe_fill": (C.c_int, [P, C.POINTER(OeDesc), C.c_uint64]),
        "gcc_sched_param_count": (C.c_uint64, []),
        "gcc_serve": (C.c_int, [P, C.POINTER(RunParams), C.POINTER(ServeParams),
                                C.POINTER(ServeResult)]),
        "gcc_sched_create": (C.c_int, [P, C.POINTER(SchedParams), C.POINTER(P)]),
        "gcc_sched_destroy": (None, [P]),
        "gcc_sched_run": (C.c_int, [P, C.POINTER(RunParams), C.POINTER(SchedResult)]),
        "gcc_sched_batches": (C.c_int, [P, P, C.c_uint64]),
        "gcc_sched_features": (C.c_int, [P, C.c_uint64, C.c_uint64, P]),
        "gcc_sched_lock_plans": (C.c_int, [P, C.c_uint64, C.c_uint64, P]),
        "gcc_sched_observe": (C.c_int, [P, C.c_uint64, C.c_uint64, C.c_int32]),
        "gcc_sched_features_var": (C.c_int, [P, C.c_uint64, C.c_uint64, P]),
        "gcc_sched_observe_var": (C.c_int, [P, C.c_uint64, C.c_uint64, C.c_int32]),
        "gcc_sched_set_weights": (C.c_int, [P, P, C.c_uint64]),
        "gcc_sched_get_weights": (C.c_int, [P, P, C.c_uint64]),
        "gcc_sched_predict": (C.c_int, [P, P, C.c_uint64, P]),
        "gcc_sched_gradient": (C.c_int, [P, P, P, C.c_uint64, P, C.POINTER(C.c_double)]),
        "gcc_sched_train": (C.c_int, [P, P, P, C.c_uint64, C.c_int32, C.POINTER(C.c_double)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


def _check(rc: int, what: str):
    if rc != 0:
        raise GccError(rc, what)


def scheme_id(name: str) -> int:
    return library().gcc_scheme_id(name.encode())


def row_bytes(layout: int) -> int:
    return library().gcc_row_bytes(layout)


def row_stride(layout: int) -> int:
    return library().gcc_row_stride(layout)


def _ptr(a: np.ndarray):
    return C.c_void_p(a.ctypes.data)


def gen_ycsb(rows: int, n_tx: int, theta: float, read_ratio: float, seed: int = 141919810,
             dedup: int = DEDUP_RESAMPLE, key_base: int = 0, threads: int = 0,
             out: np.ndarray | None = None) -> np.ndarray:
    """gen_ycsb dataset as a TX_DTYPE array (generation/gen_ycsb.cu semantics)."""
    if out is None:
        out = np.zeros(n_tx, dtype=TX_DTYPE)
    _check(library().gcc_gen_ycsb(rows, n_tx, theta, read_ratio, seed, dedup, key_base, threads,
                                  _ptr(out)), "gcc_gen_ycsb")
    return out


def gen_ycsb_var(rows: int, n_tx: int, theta: float, read_ratio: float, min_ops: int = 4,
                 max_ops: int = 64, seed: int = 141919810, key_base: int = 0, threads: int = 0):
    """Variable-length transactions: (tx_off[n_tx + 1] uint32, reqs REQ_DTYPE)."""
    lib = library()
    off = np.zeros(n_tx + 1, dtype=np.uint32)
    _check(lib.gcc_gen_ycsb_var_offsets(n_tx, min_ops, max_ops, seed, _ptr(off)),
           "gcc_gen_ycsb_var_offsets")
    reqs = np.zeros(int(off[-1]), dtype=REQ_DTYPE)
    _check(lib.gcc_gen_ycsb_var(rows, n_tx, theta, read_ratio, seed, key_base, threads,
                                _ptr(off), _ptr(reqs)), "gcc_gen_ycsb_var")
    return off, reqs


def order_entry_desc(warehouses: int = 64, districts: int = 10, customers: int = 3000,
                     items: int = 100_000, new_order_pct: int = 50, remote_line_permille: int = 10,
                     remote_customer_pct: int = 15, min_lines: int = 5, max_lines: int = 15) -> OeDesc:
    return OeDesc(warehouses, districts, customers, items, new_order_pct, remote_line_permille,
                  remote_customer_pct, min_lines, max_lines)


def gen_order_entry(desc: OeDesc, n_tx: int, seed: int = 141919810, threads: int = 0):
    """Order-entry transactions: (tx_off, reqs, kind, layout dict)."""
    lib = library()
    off = np.zeros(n_tx + 1, dtype=np.uint32)
    lay = OeLayout()
    _check(lib.gcc_oe_offsets(C.byref(desc), n_tx, seed, _ptr(off), C.byref(lay)), "gcc_oe_offsets")
    reqs = np.zeros(int(off[-1]), dtype=REQ_DTYPE)
    kind = np.zeros(n_tx, dtype=np.uint8)
    _check(lib.gcc_oe_gen(C.byref(desc), n_tx, seed, threads, _ptr(off), _ptr(reqs), _ptr(kind)),
           "gcc_oe_gen")
    return off, reqs, kind, {k: getattr(lay, k) for k, _ in OeLayout._fields_}


class Engine:
    """One table on one GPU plus its loaded transactions (gcc_engine)."""

    def __init__(self, rows: int, layout: int = LAYOUT_U64X11, index: int = INDEX_HASH,
                 fill_seed: int = 141919810, device: int = 0, max_batch: int = 65536):
        self.lib = library()
        self.rows, self.layout = rows, layout
        self.row_bytes = row_bytes(layout)
        self.row_stride = row_stride(layout)
        self.n_tx = 0
        d = TableDesc(rows, layout, index, fill_seed, device, max_batch)
        h = C.c_void_p()
        _check(self.lib.gcc_create(C.byref(d), C.byref(h)), "gcc_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self.lib.gcc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def load_txs(self, txs: np.ndarray):
        txs = np.ascontiguousarray(txs, dtype=TX_DTYPE)
        _check(self.lib.gcc_load_txs(self._h, _ptr(txs), len(txs)), "gcc_load_txs")
        self.n_tx = len(txs)

    def params(self, scheme: str, warp_density: int = 5, block_size: int = 32,
               batch_size: int = 65536, flags: int = 0, write_mode: int = WRITE_FIELD,
               write_seed: int = 1, spin_limit_ns: int = 0, backoff_ns: int = 0,
               starve_limit: int = 0, max_active: int = 0, ordered_after: int = 0) -> RunParams:
        self._scheme = scheme.encode()
        return RunParams(self._scheme, warp_density, block_size, batch_size, flags, write_mode,
                         backoff_ns, write_seed, spin_limit_ns, starve_limit, max_active,
                         ordered_after, 0)

    def run(self, scheme: str, **kw) -> dict:
        p = self.params(scheme, **kw)
        r = Result()
        rc = self.lib.gcc_run(self._h, C.byref(p), C.byref(r))
        self.last_result = r.as_dict()
        _check(rc, f"gcc_run({scheme}) err_site={r.err_site} max_attempts={r.max_attempts}")
        out = r.as_dict()
        buf = C.create_string_buffer(512)
        _check(self.lib.gcc_format_line(C.byref(p), C.byref(r), buf, 512), "gcc_format_line")
        out["line"] = buf.value.decode()
        return out

    def run_host(self, scheme: str, txs: np.ndarray, digests: np.ndarray | None = None, **kw) -> dict:
        """Run records that live in host memory (pinned for overlap): copies
        in, batches and digest copies out overlap (gcc_run_host)."""
        txs = np.ascontiguousarray(txs, dtype=TX_DTYPE)
        p = self.params(scheme, **kw)
        r = Result()
        dp = None if digests is None else _ptr(digests)
        rc = self.lib.gcc_run_host(self._h, C.byref(p), _ptr(txs), len(txs), dp, C.byref(r))
        self.last_result = r.as_dict()
        self.n_tx = len(txs)
        _check(rc, f"gcc_run_host({scheme}) err_site={r.err_site}")
        return r.as_dict()

    def run_checked(self, scheme: str, **kw) -> tuple[dict, bool]:
        """Run, then re-execute the committed transactions in their recorded
        serialization order on the GPU; returns (result, serializable)."""
        p = self.params(scheme, **kw)
        r = Result()
        v = C.c_int(-1)
        rc = self.lib.gcc_run_checked(self._h, C.byref(p), C.byref(r), C.byref(v))
        self.last_result = r.as_dict()
        _check(rc, f"gcc_run_checked({scheme})")
        return r.as_dict(), v.value == 1

    def oe_fill(self, desc: OeDesc, seed: int = 141919810):
        """Initial order-entry rows (gcc_oe_fill)."""
        _check(self.lib.gcc_oe_fill(self._h, C.byref(desc), seed), "gcc_oe_fill")

    def load_var_txs(self, tx_off: np.ndarray, reqs: np.ndarray):
        tx_off = np.ascontiguousarray(tx_off, dtype=np.uint32)
        reqs = np.ascontiguousarray(reqs, dtype=REQ_DTYPE)
        _check(self.lib.gcc_load_var_txs(self._h, _ptr(tx_off), _ptr(reqs), len(tx_off) - 1),
               "gcc_load_var_txs")
        self.n_var = len(tx_off) - 1

    def run_batches(self, scheme: str, batch_off, mode: int = BATCHES_SEQUENTIAL, **kw) -> dict:
        """Run the variable-length transactions in batches (batch_off: n+1
        transaction offsets), one launch per batch or one persistent queue."""
        boff = np.ascontiguousarray(batch_off, dtype=np.uint32)
        p = self.params(scheme, **kw)
        r = Result()
        rc = self.lib.gcc_run_batches(self._h, C.byref(p), _ptr(boff), len(boff) - 1, mode,
                                      C.byref(r))
        self.last_result = r.as_dict()
        self.n_tx = self.n_var
        self._last_nconf = 1 if mode == BATCHES_QUEUE else len(boff) - 1
        _check(rc, f"gcc_run_batches({scheme}) err_site={r.err_site}")
        return r.as_dict()

    def batch_stats(self):
        n = self._last_nconf
        wd, bs = np.zeros(n, dtype=np.int32), np.zeros(n, dtype=np.int32)
        ms = np.zeros(n, dtype=np.float64)
        _check(self.lib.gcc_get_batch_stats(self._h, _ptr(wd), _ptr(bs), _ptr(ms), n),
               "gcc_get_batch_stats")
        return wd, bs, ms

    def batch_split(self) -> np.ndarray:
        """batch_size (transactions per launch inside a batch, 0 = whole
        batch) of each entry of the last run_batches."""
        out = np.zeros(self._last_nconf, dtype=np.uint32)
        _check(self.lib.gcc_get_batch_split(self._h, _ptr(out), len(out)), "gcc_get_batch_split")
        return out

    def batch_active(self) -> np.ndarray:
        """Transactions in flight of each entry of the last run_batches."""
        a = np.zeros(self._last_nconf, dtype=np.uint64)
        _check(self.lib.gcc_get_batch_active(self._h, _ptr(a), len(a)), "gcc_get_batch_active")
        return a

    def dump_table(self) -> np.ndarray:
        a = np.empty((self.rows, self.row_bytes), dtype=np.uint8)
        _check(self.lib.gcc_dump_table(self._h, _ptr(a), a.nbytes), "gcc_dump_table")
        return a

    def upload_table(self, a: np.ndarray):
        a = np.ascontiguousarray(a, dtype=np.uint8)
        _check(self.lib.gcc_upload_table(self._h, _ptr(a), a.nbytes), "gcc_upload_table")

    def digests(self) -> np.ndarray:
        a = np.empty(self.n_tx, dtype=np.uint64)
        _check(self.lib.gcc_get_digests(self._h, _ptr(a), self.n_tx), "gcc_get_digests")
        return a

    def tx_aborts(self) -> np.ndarray:
        a = np.empty(self.n_tx, dtype=np.uint32)
        _check(self.lib.gcc_get_tx_aborts(self._h, _ptr(a), self.n_tx), "gcc_get_tx_aborts")
        return a

    def commit_log(self) -> np.ndarray:
        a = np.empty((self.n_tx, 2), dtype=np.uint64)
        _check(self.lib.gcc_get_commit_log(self._h, _ptr(a), self.n_tx), "gcc_get_commit_log")
        return a

    def read_log(self) -> np.ndarray:
        """Row images read by each (tx, op): shape (n_tx, 16, row_stride) bytes."""
        a = np.empty((self.n_tx, 16, self.row_stride), dtype=np.uint8)
        _check(self.lib.gcc_get_read_log(self._h, _ptr(a), a.nbytes), "gcc_get_read_log")
        return a

    def index_lookup(self, keys) -> np.ndarray:
        k = np.ascontiguousarray(keys, dtype=np.uint32)
        r = np.empty_like(k)
        _check(self.lib.gcc_index_lookup(self._h, _ptr(k), _ptr(r), len(k)), "gcc_index_lookup")
        return r

    def last_kernel_ms(self):
        ms, n = C.c_double(), C.c_uint64()
        _check(self.lib.gcc_last_kernel_ms(self._h, C.byref(ms), C.byref(n)), "gcc_last_kernel_ms")
        return ms.value, n.value


class Scheduler:
    """Learned contention scheduling over an Engine's loaded 16-request
    records (gcc_sched_*): a BF16 MLP predicts which transactions abort under
    plain ordering; scheduled batches defer those into a capped sub-batch.
    mode=SCHED_PLAIN runs every batch with plain ordering through the same
    driver (the comparison arm)."""

    def __init__(self, engine: "Engine", mode: int = SCHED_LEARNED, explore_every: int = 0,
                 probe_rows: int = 0, train_steps: int = 0, minibatch: int = 0, lr: float = 0.0,
                 defer_threshold: float = 0.0, fixed_arm: int = 0, min_sched: int = 0,
                 seed: int = 1, plan_threshold: int = 0, plan_after: int = 0):
        self.engine = engine
        self.lib = engine.lib
        self._h = C.c_void_p()
        prm = SchedParams(mode, explore_every, probe_rows, train_steps, minibatch, lr,
                          defer_threshold, fixed_arm, min_sched, plan_threshold, seed,
                          plan_after, 0)
        _check(self.lib.gcc_sched_create(engine._h, C.byref(prm), C.byref(self._h)),
               "gcc_sched_create")
        self.n_params = int(self.lib.gcc_sched_param_count())
        self._nb = 0

    def close(self):
        if self._h:
            self.lib.gcc_sched_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def run(self, scheme: str, **kw) -> dict:
        p = self.engine.params(scheme, **kw)
        r = SchedResult()
        rc = self.lib.gcc_sched_run(self._h, C.byref(p), C.byref(r))
        out = {k: getattr(r, k) for k, _ in SchedResult._fields_ if k != "run"}
        out.update(r.run.as_dict())
        self.last_result = out
        n = self.engine.n_tx
        self._nb = (n + p.batch_size - 1) // p.batch_size
        self.engine.n_tx = n
        _check(rc, f"gcc_sched_run({scheme}) err_site={r.run.err_site}")
        return out

    def serve(self, scheme: str, rate_tps: float, seed: int = 1, max_batch: int = 0,
              min_batch: int = 0, max_wait_us: float = 0.0, **kw) -> dict:
        """Serve the engine's loaded variable-length transactions as a Poisson
        arrival stream (gcc_serve); latencies are arrival -> commit."""
        p = self.engine.params(scheme, **kw)
        sp = ServeParams(rate_tps, seed, max_batch, min_batch, max_wait_us)
        r = ServeResult()
        rc = self.lib.gcc_serve(self._h, C.byref(p), C.byref(sp), C.byref(r))
        out = {k: getattr(r, k) for k, _ in ServeResult._fields_}
        self.last_result = out
        self._nb = int(r.batches)
        self.engine.n_tx = self.engine.n_var
        _check(rc, f"gcc_serve({scheme})")
        return out

    def batches(self) -> list[dict]:
        arr = (SchedBatch * self._nb)()
        _check(self.lib.gcc_sched_batches(self._h, arr, self._nb), "gcc_sched_batches")
        return [{k: getattr(b, k) for k, _ in SchedBatch._fields_} for b in arr]

    def features(self, first: int, n: int) -> np.ndarray:
        out = np.zeros((n, SCHED_FEAT_STRIDE), dtype=np.uint16)
        _check(self.lib.gcc_sched_features(self._h, first, n, _ptr(out)), "gcc_sched_features")
        return out

    def lock_plans(self, first: int, n: int) -> np.ndarray:
        """2PL lock plans (u64 per record) of records first .. first+n-1
        against the current frequency table (gcc_sched_lock_plans)."""
        out = np.zeros(n, dtype=np.uint64)
        _check(self.lib.gcc_sched_lock_plans(self._h, first, n, _ptr(out)), "gcc_sched_lock_plans")
        return out

    def features_var(self, first: int, n: int) -> np.ndarray:
        out = np.zeros((n, SCHED_FEAT_STRIDE), dtype=np.uint16)
        _check(self.lib.gcc_sched_features_var(self._h, first, n, _ptr(out)), "gcc_sched_features_var")
        return out

    def observe_var(self, first: int, n: int, clear: bool = False):
        _check(self.lib.gcc_sched_observe_var(self._h, first, n, 1 if clear else 0),
               "gcc_sched_observe_var")

    def observe(self, first: int, n: int, clear: bool = False):
        _check(self.lib.gcc_sched_observe(self._h, first, n, 1 if clear else 0), "gcc_sched_observe")

    def set_weights(self, w: np.ndarray):
        w = np.ascontiguousarray(w, dtype=np.float32)
        _check(self.lib.gcc_sched_set_weights(self._h, _ptr(w), len(w)), "gcc_sched_set_weights")

    def get_weights(self) -> np.ndarray:
        w = np.zeros(self.n_params, dtype=np.float32)
        _check(self.lib.gcc_sched_get_weights(self._h, _ptr(w), len(w)), "gcc_sched_get_weights")
        return w

    def predict(self, feat: np.ndarray) -> np.ndarray:
        feat = np.ascontiguousarray(feat, dtype=np.uint16)
        p = np.zeros(len(feat), dtype=np.float32)
        _check(self.lib.gcc_sched_predict(self._h, _ptr(feat), len(feat), _ptr(p)), "gcc_sched_predict")
        return p

    def gradient(self, feat: np.ndarray, labels: np.ndarray):
        feat = np.ascontiguousarray(feat, dtype=np.uint16)
        y = np.ascontiguousarray(labels, dtype=np.uint8)
        g = np.zeros(self.n_params, dtype=np.float32)
        loss = C.c_double()
        _check(self.lib.gcc_sched_gradient(self._h, _ptr(feat), _ptr(y), len(feat), _ptr(g),
                                           C.byref(loss)), "gcc_sched_gradient")
        return g, loss.value

    def train(self, feat: np.ndarray, labels: np.ndarray, steps: int) -> float:
        feat = np.ascontiguousarray(feat, dtype=np.uint16)
        y = np.ascontiguousarray(labels, dtype=np.uint8)
        loss = C.c_double()
        _check(self.lib.gcc_sched_train(self._h, _ptr(feat), _ptr(y), len(feat), steps,
                                        C.byref(loss)), "gcc_sched_train")
        return loss.value
