"""GPU parity of every CC scheme against the CPU oracle, through the C ABI.

Bar (integer, bit-exact):
  * deterministic schemes (gacco, gputx): final table bytes and per-tx read
    digests equal the oracle's serial execution in the scheme's own order
    (gacco: tx index within each batch, include/gacco.cuh:156-175; gputx:
    (rank, tx) with the rank function of src/gputx.cu:17-27);
  * all other schemes: replaying the committed transactions serially in the
    recorded commit order reproduces the final table and every read digest
    (and, where enabled, every read row image).
"""
import numpy as np
import pytest

import gpu_cc_tb_b200 as g

pytestmark = pytest.mark.gpu

SPIN_NS = 2_000_000_000
NONDET = [s for s in g.SCHEMES if s not in ("gacco", "gputx")]


def expected_order(oracle, scheme, eng, txs, rows):
    if scheme == "gacco":
        return np.arange(len(txs), dtype=np.uint32)
    if scheme == "gputx":
        return oracle.gputx_order(txs, rows)[1]
    return oracle.commit_order(eng.commit_log())


def run_and_check(oracle, eng, init, txs, scheme, wd, bs, batch, write_mode, layout,
                  write_seed=99, read_log=False, extra_flags=0, **kw):
    eng.upload_table(init)
    flags = g.F_COMMIT_LOG | (g.F_READ_LOG if read_log else 0) | extra_flags
    res = eng.run(scheme, warp_density=wd, block_size=bs, batch_size=batch, flags=flags,
                  write_mode=write_mode, write_seed=write_seed, spin_limit_ns=SPIN_NS, **kw)
    assert res["committed"] == len(txs)
    table = eng.dump_table()
    dg = eng.digests()
    order = expected_order(oracle, scheme, eng, txs, eng.rows)
    assert sorted(order.tolist()) == list(range(len(txs)))
    ref_t, ref_dg, ref_rl = oracle.replay(init, layout, txs, order, write_mode, write_seed,
                                          read_log=read_log)
    bad_rows = np.nonzero((table != ref_t).any(axis=1))[0]
    assert len(bad_rows) == 0, f"{scheme} wd={wd}: {len(bad_rows)} rows differ, e.g. {bad_rows[:8]}"
    bad_tx = np.nonzero(dg != ref_dg)[0]
    assert len(bad_tx) == 0, f"{scheme} wd={wd}: {len(bad_tx)} digests differ, e.g. {bad_tx[:8]}"
    if read_log:
        rl = eng.read_log()
        rb = eng.row_bytes
        for t in range(len(txs)):
            n = int(txs[t]["request_cnt"])
            for i in range(n):
                if txs[t]["requests"][i]["read"]:
                    assert np.array_equal(rl[t, i, :rb], ref_rl[t, i, :rb]), (scheme, t, i)
    return res


@pytest.fixture(scope="module")
def small_u64(oracle):
    rows, layout = 65536, g.LAYOUT_U64X11
    txs = g.gen_ycsb(rows, 8192, 0.6, 0.8, seed=11, dedup=g.DEDUP_RESAMPLE, key_base=0)
    init = oracle.fill_table(rows, layout, 141919810)
    eng = g.Engine(rows, layout=layout, index=g.INDEX_HASH, fill_seed=141919810, max_batch=2048)
    eng.load_txs(txs)
    assert np.array_equal(eng.dump_table(), init), "table fill differs from oracle"
    yield eng, init, txs
    eng.close()


@pytest.mark.parametrize("wd", [0, 3, 5])
@pytest.mark.parametrize("scheme", g.SCHEMES)
def test_scheme_parity_field_writes(oracle, small_u64, scheme, wd):
    eng, init, txs = small_u64
    run_and_check(oracle, eng, init, txs, scheme, wd, 4, 2048, g.WRITE_FIELD, g.LAYOUT_U64X11)


@pytest.fixture(scope="module")
def small_ref104(oracle):
    # the reference's own format: 104-byte Item rows, dropped duplicate keys,
    # keys in [1, rows-1], sorted-array index, whole-row copies on write
    rows, layout = 2048, g.LAYOUT_REF104
    txs = g.gen_ycsb(rows, 4096, 0.6, 0.5, seed=5, dedup=g.DEDUP_DROP, key_base=1)
    init = oracle.fill_table(rows, layout, 77)
    eng = g.Engine(rows, layout=layout, index=g.INDEX_SORTED, fill_seed=77, max_batch=1024)
    eng.load_txs(txs)
    assert np.array_equal(eng.dump_table(), init)
    yield eng, init, txs
    eng.close()


@pytest.mark.parametrize("scheme", g.SCHEMES)
def test_scheme_parity_rowcopy_ref104(oracle, small_ref104, scheme):
    eng, init, txs = small_ref104
    run_and_check(oracle, eng, init, txs, scheme, 5, 32, 1024, g.WRITE_ROWCOPY, g.LAYOUT_REF104,
                  read_log=True)


@pytest.mark.parametrize("scheme", g.SCHEMES)
def test_scheme_parity_hot_rows(oracle, scheme):
    # theta = 0.99 over 64 rows: most transactions conflict
    rows, layout = 64, g.LAYOUT_U64X11
    txs = g.gen_ycsb(rows, 2048, 0.99, 0.5, seed=3, dedup=g.DEDUP_RESAMPLE, key_base=0)
    init = oracle.fill_table(rows, layout, 9)
    with g.Engine(rows, layout=layout, index=g.INDEX_DIRECT, fill_seed=9, max_batch=512) as eng:
        eng.load_txs(txs)
        res = run_and_check(oracle, eng, init, txs, scheme, 5, 8, 512, g.WRITE_FIELD, layout)
    if scheme == "gputx":
        _, _, mx = oracle.gputx_order(txs, rows)
        assert res["rank_count"] == mx + 1


@pytest.mark.parametrize("scheme", ["tpl_nw", "tpl_wd", "to", "mvcc", "silo", "tictoc"])
def test_starvation_control_and_in_flight_cap(oracle, scheme):
    # hot rows with an aggressive starvation limit (admission pause after 2
    # aborts, one-at-a-time retries after 8) and with few transactions in
    # flight: neither may change what commits or the serial equivalence
    rows, layout = 64, g.LAYOUT_U64X11
    txs = g.gen_ycsb(rows, 2048, 0.99, 0.5, seed=31, dedup=g.DEDUP_RESAMPLE, key_base=0)
    init = oracle.fill_table(rows, layout, 9)
    with g.Engine(rows, layout=layout, index=g.INDEX_DIRECT, fill_seed=9, max_batch=1024) as eng:
        eng.load_txs(txs)
        run_and_check(oracle, eng, init, txs, scheme, 5, 32, 1024, g.WRITE_FIELD, layout,
                      starve_limit=2)
        run_and_check(oracle, eng, init, txs, scheme, 3, 8, 1024, g.WRITE_FIELD, layout,
                      max_active=40)


@pytest.mark.parametrize("scheme", ["tpl_nw", "tpl_wd", "slow_tpl_nw", "slow_tpl_wd", "to",
                                    "slow_to"])
@pytest.mark.parametrize("order_flag,ordered_after", [(0, 1), (0, 3), (g.F_REQUEST_ORDER, 1),
                                                      (g.F_REQUEST_ORDER, 0)])
def test_retry_orders(oracle, scheme, order_flag, ordered_after):
    # 2PL / TO retries that visit their requests one at a time (from the
    # first retry, or after a few), with the failed request last (default)
    # or in request order (the reference's order): only the order of the
    # accesses changes, so every run replays bit-exactly
    rows, layout = 64, g.LAYOUT_U64X11
    txs = g.gen_ycsb(rows, 2048, 0.99, 0.5, seed=17, dedup=g.DEDUP_RESAMPLE, key_base=0)
    init = oracle.fill_table(rows, layout, 9)
    with g.Engine(rows, layout=layout, index=g.INDEX_DIRECT, fill_seed=9, max_batch=1024) as eng:
        eng.load_txs(txs)
        res = run_and_check(oracle, eng, init, txs, scheme, 5, 8, 1024, g.WRITE_FIELD, layout,
                            ordered_after=ordered_after, extra_flags=order_flag)
        assert res["aborts"] > 0


@pytest.mark.parametrize("scheme", ["tpl_nw", "tictoc", "gacco", "mvcc"])
def test_rowcopy_u64_with_read_log(oracle, scheme):
    rows, layout = 1024, g.LAYOUT_U64X11
    txs = g.gen_ycsb(rows, 2048, 0.7, 0.6, seed=21, dedup=g.DEDUP_RESAMPLE, key_base=0)
    init = oracle.fill_table(rows, layout, 5)
    with g.Engine(rows, layout=layout, index=g.INDEX_HASH, fill_seed=5, max_batch=700) as eng:
        eng.load_txs(txs)
        run_and_check(oracle, eng, init, txs, scheme, 2, 2, 700, g.WRITE_ROWCOPY, layout,
                      read_log=True)


def test_gacco_and_gputx_commit_keys(oracle):
    rows, layout = 512, g.LAYOUT_U64X11
    txs = g.gen_ycsb(rows, 3000, 0.9, 0.5, seed=8, dedup=g.DEDUP_RESAMPLE, key_base=0)
    with g.Engine(rows, layout=layout, index=g.INDEX_HASH, fill_seed=1, max_batch=1000) as eng:
        eng.load_txs(txs)
        eng.run("gacco", warp_density=5, block_size=4, batch_size=1000, flags=g.F_COMMIT_LOG,
                spin_limit_ns=SPIN_NS)
        log = eng.commit_log()
        assert np.array_equal(log[:, 0], np.arange(len(txs)))
        eng.run("gputx", warp_density=5, block_size=4, batch_size=1000, flags=g.F_COMMIT_LOG,
                spin_limit_ns=SPIN_NS)
        log = eng.commit_log()
        _, order, _ = oracle.gputx_order(txs, rows)
        pos = np.empty(len(txs), dtype=np.uint64)
        pos[order] = np.arange(len(txs))
        assert np.array_equal(log[:, 0], pos)


def test_edge_cases_empty_single_and_full(oracle):
    rows, layout = 256, g.LAYOUT_U64X11
    txs = np.zeros(64, dtype=g.TX_DTYPE)
    for t in range(64):
        n = [0, 1, 16, 16][t % 4]
        txs[t]["request_cnt"] = n
        keys = np.sort(np.random.default_rng(t).choice(rows, size=n, replace=False))
        for i in range(n):
            txs[t]["requests"][i] = (1 if (t % 4 != 3) and (i % 2 == 0) else 0, keys[i])
    init = oracle.fill_table(rows, layout, 4)
    with g.Engine(rows, layout=layout, index=g.INDEX_HASH, fill_seed=4, max_batch=64) as eng:
        eng.load_txs(txs)
        for scheme in g.SCHEMES:
            run_and_check(oracle, eng, init, txs, scheme, 4, 1, 64, g.WRITE_FIELD, layout)


def test_errors_are_reported_not_hung(oracle):
    rows = 128
    with g.Engine(rows, layout=g.LAYOUT_U64X11, index=g.INDEX_HASH, fill_seed=1, max_batch=16) as eng:
        bad = np.zeros(4, dtype=g.TX_DTYPE)
        bad[1]["request_cnt"] = 17
        eng.load_txs(bad)
        with pytest.raises(g.GccError) as ei:
            eng.run("tpl_nw", warp_density=5, block_size=1, batch_size=16)
        assert ei.value.status == -5  # GCC_EFORMAT
        miss = np.zeros(4, dtype=g.TX_DTYPE)
        miss[2]["request_cnt"] = 1
        miss[2]["requests"][0] = (1, 1000)  # key not in the table
        eng.load_txs(miss)
        with pytest.raises(g.GccError) as ei:
            eng.run("silo", warp_density=5, block_size=1, batch_size=16)
        assert ei.value.status == -6  # GCC_EKEY
        eng.load_txs(np.zeros(2, dtype=g.TX_DTYPE))
        for kw in (dict(warp_density=6), dict(block_size=0), dict(block_size=33),
                   dict(batch_size=0)):
            with pytest.raises(g.GccError) as ei:
                eng.run("tpl_nw", **kw)
            assert ei.value.status == -1
        with pytest.raises(g.GccError):
            eng.run("no_such_scheme")


@pytest.mark.parametrize("index", [g.INDEX_HASH, g.INDEX_SORTED, g.INDEX_DIRECT])
def test_index_lookup(index):
    rows = 100_000
    with g.Engine(rows, layout=g.LAYOUT_U64X11, index=index, fill_seed=2) as eng:
        keys = np.concatenate([np.arange(rows, dtype=np.uint32),
                               np.array([rows, rows + 7, 2**32 - 2], dtype=np.uint32)])
        got = eng.index_lookup(keys)
        assert np.array_equal(got[:rows], np.arange(rows, dtype=np.uint32))
        assert (got[rows:] == 0xFFFFFFFF).all()
