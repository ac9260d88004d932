"""C-ABI surface checks that need no GPU: the library loads, exports every
symbol declared in include/gcc_engine.h, and its host-only entry points
(scheme names, layouts, generator, result line) behave like the reference's
(benchmark_cpu/ycsb.cu:89-195, include/runtime.cuh:182-196)."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

import gpu_cc_tb_b200 as g

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    hdr = (ROOT / "include" / "gcc_engine.h").read_text()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return sorted(set(re.findall(r"\b(gcc_[a-z_0-9]+)\s*\(", hdr)))


def test_library_exports_every_declared_symbol(gcc):
    syms = declared_symbols()
    assert len(syms) >= 20
    out = subprocess.run(["nm", "-D", "--defined-only", str(g.library_path())],
                         capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (gcc_[a-z_0-9]+)", out))
    missing = [s for s in syms if s not in exported]
    assert not missing, missing
    lib = g.library()
    for s in syms:
        assert hasattr(lib, s)


def test_scheme_names_and_aliases(gcc):
    ids = [g.scheme_id(s) for s in g.SCHEMES]
    assert ids == list(range(14))
    assert g.scheme_id("slowto") == g.scheme_id("slow_to")
    assert g.scheme_id("slowmvcc") == g.scheme_id("slow_mvcc")
    assert g.scheme_id("nope") == -1
    assert g.library().gcc_scheme_id(None) == -1


def test_layouts(gcc):
    assert (g.row_bytes(g.LAYOUT_U64X11), g.row_stride(g.LAYOUT_U64X11)) == (88, 96)
    assert (g.row_bytes(g.LAYOUT_REF104), g.row_stride(g.LAYOUT_REF104)) == (104, 112)
    assert g.TX_DTYPE.itemsize == 136


def test_strerror(gcc):
    lib = g.library()
    for code in range(0, -10, -1):
        assert lib.gcc_strerror(code).decode()
    assert lib.gcc_version().decode().startswith("gpu_cc_tb_b200")


@pytest.mark.parametrize("dedup,key_base", [(g.DEDUP_DROP, 1), (g.DEDUP_RESAMPLE, 0)])
def test_generator_matches_oracle_restatement(gcc, oracle, dedup, key_base):
    a = g.gen_ycsb(5000, 3000, 0.8, 0.9, seed=123, dedup=dedup, key_base=key_base, threads=3)
    b = oracle.gen_ycsb(5000, 3000, 0.8, 0.9, 123, dedup, key_base)
    assert np.array_equal(a.view(np.uint8), b.view(np.uint8))
    # independent of the host thread count
    c = g.gen_ycsb(5000, 3000, 0.8, 0.9, seed=123, dedup=dedup, key_base=key_base, threads=1)
    assert np.array_equal(a.view(np.uint8), c.view(np.uint8))


def test_generator_format_rules(gcc):
    rows = 1000
    a = g.gen_ycsb(rows, 4000, 0.9, 0.75, seed=1, dedup=g.DEDUP_DROP, key_base=1)
    cnt = a["request_cnt"]
    assert cnt.max() <= 16 and cnt.min() >= 1
    reads = 0
    for t in range(len(a)):
        k = a[t]["requests"]["key"][: cnt[t]]
        assert (np.diff(k.astype(np.int64)) > 0).all()  # sorted, distinct
        assert k.min() >= 1 and k.max() <= rows - 1     # gen_ycsb key range
        assert (a[t]["requests"][cnt[t]:]["key"] == 0).all()
        reads += a[t]["requests"]["read"][: cnt[t]].sum()
    assert abs(reads / cnt.sum() - 0.75) < 0.02
    r = g.gen_ycsb(rows, 4000, 0.9, 0.75, seed=1, dedup=g.DEDUP_RESAMPLE, key_base=0)
    assert (r["request_cnt"] == 16).all()


def test_generator_rejects_bad_arguments(gcc):
    lib = g.library()
    out = np.zeros(1, dtype=g.TX_DTYPE)
    p = C.c_void_p(out.ctypes.data)
    assert lib.gcc_gen_ycsb(100, 1, 1.0, 0.5, 1, 0, 1, 1, p) == -1   # theta = 1
    assert lib.gcc_gen_ycsb(100, 1, 0.5, 1.5, 1, 0, 1, 1, p) == -1   # ratio > 1
    assert lib.gcc_gen_ycsb(2, 1, 0.5, 0.5, 1, 0, 1, 1, p) == -1     # too few rows
    assert lib.gcc_gen_ycsb(100, 1, 0.5, 0.5, 1, 7, 1, 1, p) == -1   # dedup mode


def test_result_line_format(gcc):
    lib = g.library()
    p = g.RunParams(b"tpl_nw", 5, 32, 65536, 0, 0, 0, 1, 0)  # backoff 0, seed 1
    r = g.Result()
    r.tx_per_s, r.aborts, r.tot_s, r.pre_s, r.proc_s = 18670000.0, 15736673, 0.0561, 0.001, 0.05
    r.ts_d, r.wait_d, r.abort_d, r.mng_d, r.tot_d, r.idx_d = 0, 1e-4, 0.5, 0.25, 0.183, 0.085
    buf = C.create_string_buffer(256)
    assert lib.gcc_format_line(C.byref(p), C.byref(r), buf, 256) == 0
    cols = buf.value.decode().split(",")
    assert len(cols) == 15
    assert cols[:4] == ["tpl_nw", "5", "32", "65536"]
    assert cols[4] == "1.867e+07" and cols[5] == "15736673"   # std::ostream float style
    assert cols[11] == "0.085" and cols[14] == "0.0561"


def test_create_without_gpu_fails_cleanly(gcc):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("GPU present")
    except ImportError:
        pass
    lib = g.library()
    d = g.TableDesc(1024, 0, 0, 1, 0, 1024)
    h = C.c_void_p()
    assert lib.gcc_create(C.byref(d), C.byref(h)) == -9  # GCC_ENODEV
    assert lib.gcc_load_txs(None, None, 0) == -1
    assert lib.gcc_run(None, None, None) == -1


def test_variable_length_generator_rules(gcc):
    off, reqs = g.gen_ycsb_var(5000, 3000, 0.8, 0.9, min_ops=4, max_ops=64, seed=3, threads=3)
    cnt = np.diff(off.astype(np.int64))
    assert cnt.min() >= 4 and cnt.max() <= 64
    assert abs(cnt.mean() - 34) < 2
    for t in range(0, 3000, 37):
        k = reqs["key"][off[t]:off[t + 1]].astype(np.int64)
        assert (np.diff(k) > 0).all() and k.max() < 5000
    off2, reqs2 = g.gen_ycsb_var(5000, 3000, 0.8, 0.9, min_ops=4, max_ops=64, seed=3, threads=1)
    assert np.array_equal(off, off2) and np.array_equal(reqs.view(np.uint8), reqs2.view(np.uint8))
    assert abs(reqs["read"].mean() - 0.9) < 0.01
