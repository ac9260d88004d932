"""gcc_run_tpl_nw_noalloc: the 2PL no-wait run for callers that cannot call
cudaMalloc (their device memory belongs to another allocator, or they run on a
thread where cudaMalloc's implicit device synchronisation is not acceptable).
It takes every input and output as a caller-owned device buffer and keeps its
scratch in a static device array of the library.

Checked through the C ABI against the existing entry point (gcc_run with
tpl_nw) on the same inputs, bit-exact, on two calls in a row. The
transactions of that case touch disjoint rows, so the result does not depend
on the order in which they commit and both entry points must agree byte for
byte. A second case is contended (Zipf theta 0.99 over 4,096 rows, half the
requests writes): the commit order then differs from run to run, so it
checks what every serial order must give -- all transactions commit, some
abort on the way, every field ends with the initial value or a value some
transaction wrote to that field, rows nobody writes keep their bytes, and
transactions that read only such rows return the oracle's digests -- on two
calls in a row, the second starting from the lock words and counters the
first left behind. This file is named to be collected last."""
import ctypes as C

import numpy as np
import pytest

import gpu_cc_tb_b200 as g

pytestmark = pytest.mark.gpu

ROWS = 1 << 20          # the entry point's stated maximum
N_TX = 32768


def disjoint_txs(n, seed):
    rng = np.random.default_rng(seed)
    txs = np.zeros(n, dtype=g.TX_DTYPE)
    txs["request_cnt"] = 16
    keys = (np.arange(n, dtype=np.uint32)[:, None] * 16 + np.arange(16, dtype=np.uint32)[None, :])
    txs["requests"]["key"] = keys
    txs["requests"]["read"] = (rng.random((n, 16)) < 0.7).astype(np.int32)
    return txs


def bind(lib):
    fn = lib.gcc_run_tpl_nw_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p,
                   C.c_uint64, C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
    return fn


def test_no_alloc_matches_existing_entry_point_twice():
    import torch

    lib = g.library()
    noalloc = bind(lib)
    txs = disjoint_txs(N_TX, 1)
    stride, rb = g.row_stride(g.LAYOUT_U64X11), g.row_bytes(g.LAYOUT_U64X11)

    with g.Engine(ROWS, layout=g.LAYOUT_U64X11, index=g.INDEX_HASH, fill_seed=77,
                  max_batch=N_TX) as eng:
        table0 = eng.dump_table()
        eng.load_txs(txs)
        refs = []
        for seed in (11, 12):
            eng.run("tpl_nw", warp_density=5, block_size=32, batch_size=N_TX, write_seed=seed)
            refs.append((eng.dump_table(), eng.digests()))

    # caller-owned device buffers
    dev = torch.device("cuda", 0)
    padded = np.zeros((ROWS, stride), dtype=np.uint8)
    padded[:, :rb] = table0
    table_d = torch.from_numpy(padded.reshape(-1)).to(dev)
    txs_d = torch.from_numpy(txs.view(np.uint8).copy()).to(dev)
    dig_d = torch.zeros(N_TX, dtype=torch.int64, device=dev)
    ab_d = torch.zeros(N_TX, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    for (ref_t, ref_dg), seed in zip(refs, (11, 12)):
        committed, aborts = C.c_uint64(), C.c_uint64()
        rc = noalloc(txs_d.data_ptr(), N_TX, table_d.data_ptr(), ROWS, dig_d.data_ptr(),
                     ab_d.data_ptr(), seed, None, C.byref(committed), C.byref(aborts))
        assert rc == 0, g.GccError(rc, "gcc_run_tpl_nw_noalloc")
        assert committed.value == N_TX and aborts.value == 0
        got_t = table_d.cpu().numpy().reshape(ROWS, stride)[:, :rb]
        got_dg = dig_d.cpu().numpy().view(np.uint64)
        assert np.array_equal(got_t, ref_t)
        assert np.array_equal(got_dg, ref_dg)
        assert (ab_d.cpu().numpy() == 0).all()


def test_no_alloc_rejects_sizes_beyond_its_limit():
    lib = g.library()
    noalloc = bind(lib)
    # rejected before any device work
    assert noalloc(C.c_void_p(16), 1, C.c_void_p(16), ROWS + 1, C.c_void_p(16), C.c_void_p(16),
                   1, None, None, None) == -1
    assert noalloc(None, 1, None, 16, None, None, 1, None, None, None) == -1


def test_no_alloc_contended_two_calls(oracle):
    import torch

    lib = g.library()
    noalloc = bind(lib)
    rows, n = 4096, 16384
    stride, rb = g.row_stride(g.LAYOUT_U64X11), g.row_bytes(g.LAYOUT_U64X11)
    txs = g.gen_ycsb(rows, n, 0.99, 0.5, seed=5, dedup=g.DEDUP_RESAMPLE, key_base=0)
    init = oracle.fill_table(rows, g.LAYOUT_U64X11, 3)
    cnt = txs["request_cnt"].astype(np.int64)
    valid = np.arange(16)[None, :] < cnt[:, None]
    keys = txs["requests"]["key"].astype(np.int64)
    isw = valid & (txs["requests"]["read"] == 0)

    dev = torch.device("cuda", 0)
    padded = np.zeros((rows, stride), dtype=np.uint8)
    padded[:, :rb] = init
    table_d = torch.from_numpy(padded.reshape(-1)).to(dev)
    txs_d = torch.from_numpy(txs.view(np.uint8).copy()).to(dev)
    dig_d = torch.zeros(n, dtype=torch.int64, device=dev)
    ab_d = torch.zeros(n, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()

    state = init.copy()
    for seed in (21, 22):
        committed, aborts = C.c_uint64(), C.c_uint64()
        rc = noalloc(txs_d.data_ptr(), n, table_d.data_ptr(), rows, dig_d.data_ptr(),
                     ab_d.data_ptr(), seed, None, C.byref(committed), C.byref(aborts))
        assert rc == 0, g.GccError(rc, "gcc_run_tpl_nw_noalloc")
        assert committed.value == n
        assert aborts.value > 0, "the contended case should abort"
        assert int(ab_d.cpu().numpy().astype(np.int64).sum()) == aborts.value
        got = table_d.cpu().numpy().reshape(rows, stride)[:, :rb]
        words = got.view(np.uint64)            # [rows, 11]: key, then 10 fields
        before = state.view(np.uint64)
        # every (row, field) ends with its value before the call or with a
        # value some transaction of this call wrote to it
        written = {}
        for t, i in zip(*np.nonzero(isw)):
            f = oracle.write_field(seed, int(t), int(i))
            written.setdefault((int(keys[t, i]), f), set()).add(oracle.write_value(seed, int(t), int(i)))
        for r in range(rows):
            for f in range(10):
                v = int(words[r, 1 + f])
                ok = written.get((r, f))
                if ok is None:
                    assert v == int(before[r, 1 + f]), (r, f)
                else:
                    assert v in ok, (r, f)
            assert int(words[r, 0]) == int(before[r, 0])
        # transactions that read only rows nobody writes see fixed images
        wrows = np.zeros(rows, dtype=bool)
        wrows[keys[isw]] = True
        quiet = [t for t in range(n) if not wrows[keys[t][valid[t]]].any()]
        if quiet:
            qtx = txs[quiet]
            _, ref_dg, _ = oracle.replay(state, g.LAYOUT_U64X11, qtx,
                                         np.arange(len(qtx), dtype=np.uint32), g.WRITE_FIELD, seed)
            got_dg = dig_d.cpu().numpy().view(np.uint64)[quiet]
            # replay numbers the quiet transactions 0..k-1; their digests do
            # not depend on the transaction id (reads only)
            assert np.array_equal(got_dg, ref_dg)
        state = got.copy()
