"""GPU parity at the sizes the benchmark runs, through the C ABI.

The small-case matrix (test_gpu_parity.py) cannot show that the memory
ordering of the schemes holds when a full B200 of transactions is in flight:
persistent grids hold 148 x 1,024 threads, i.e. 4,736 transactions at
warp_density 5, and a batch of 65,536 keeps them busy. These cases run the
real shapes and apply the same bar:

  * gacco / gputx: final table bytes and every read digest equal the
    oracle's serial execution in the scheme's own order (gacco: tx index
    within each batch, include/gacco.cuh:156-175; gputx: (rank, tx),
    src/gputx.cu:17-27);
  * every other scheme: replaying the committed transactions one by one in
    the recorded commit order reproduces the final table byte for byte and
    every read digest (the serializability bar of src/runtime.cu:129-158,
    checked on values rather than on the conflict graph).

Shapes:
  * the 1,048,576-row YCSB point: 1,048,576 rows of u64 key + 10 u64 fields,
    65,536 transactions of 16 requests, Zipf theta 0.1, read ratio 0.9,
    batch 65,536, warp_density 5, block_size 32;
  * the benchmark's plain shape: 10,485,760 rows, theta 0.6, read ratio 0.9,
    65,536-transaction batches (4 of them), warp_density 5, block_size 32,
    per-batch launches and the device-queue launch (GCC_F_QUEUE);
  * high contention on the same table: theta 0.99, 2 batches, with the
    default persistent grid and with 512 transactions in flight.
"""
import numpy as np
import pytest

import gpu_cc_tb_b200 as g

pytestmark = pytest.mark.gpu

SPIN_NS = 4_000_000_000
LAYOUT = g.LAYOUT_U64X11
SEED = 141919810


def check(oracle, eng, init, txs, scheme, res, write_seed):
    assert res["committed"] == len(txs)
    if scheme == "gacco":
        order = np.arange(len(txs), dtype=np.uint32)
    elif scheme == "gputx":
        order = oracle.gputx_order(txs, eng.rows)[1]
    else:
        order = oracle.commit_order(eng.commit_log())
    assert len(order) == len(txs)
    ref_t, ref_dg, _ = oracle.replay(init, LAYOUT, txs, order, g.WRITE_FIELD, write_seed)
    dg = eng.digests()
    bad_tx = np.nonzero(dg != ref_dg)[0]
    assert len(bad_tx) == 0, f"{scheme}: {len(bad_tx)} digests differ, e.g. {bad_tx[:8]}"
    table = eng.dump_table()
    if not np.array_equal(table, ref_t):
        bad = np.nonzero((table != ref_t).any(axis=1))[0]
        raise AssertionError(f"{scheme}: {len(bad)} rows differ, e.g. {bad[:8]}")


def run(eng, init, scheme, batch, flags=0, write_seed=7, **kw):
    eng.upload_table(init)
    return eng.run(scheme, warp_density=5, block_size=32, batch_size=batch,
                   flags=g.F_COMMIT_LOG | flags, write_mode=g.WRITE_FIELD,
                   write_seed=write_seed, spin_limit_ns=SPIN_NS, **kw)


# ---- the 1,048,576-row point -----------------------------------------------

@pytest.fixture(scope="module")
def rows_1m(oracle):
    rows = 1_048_576
    txs = g.gen_ycsb(rows, 65_536, 0.1, 0.9, seed=SEED, dedup=g.DEDUP_RESAMPLE, key_base=0)
    init = oracle.fill_table(rows, LAYOUT, SEED)
    eng = g.Engine(rows, layout=LAYOUT, index=g.INDEX_HASH, fill_seed=SEED, max_batch=65_536)
    eng.load_txs(txs)
    assert np.array_equal(eng.dump_table(), init)
    yield eng, init, txs
    eng.close()


@pytest.mark.parametrize("scheme", g.SCHEMES)
def test_1m_rows_theta01_one_batch(oracle, rows_1m, scheme):
    eng, init, txs = rows_1m
    res = run(eng, init, scheme, 65_536)
    assert res["batches"] == 1
    check(oracle, eng, init, txs, scheme, res, 7)


def test_1m_rows_theta01_queue(oracle, rows_1m):
    eng, init, txs = rows_1m
    res = run(eng, init, "tpl_nw", 8_192, flags=g.F_QUEUE)
    assert res["batches"] == 1  # eight batches, one launch
    check(oracle, eng, init, txs, "tpl_nw", res, 7)


# ---- the benchmark's 10,485,760-row table ----------------------------------

BIG_ROWS = 10_485_760
BATCH = 65_536


@pytest.fixture(scope="module")
def big_table(oracle):
    init = oracle.fill_table(BIG_ROWS, LAYOUT, SEED)
    eng = g.Engine(BIG_ROWS, layout=LAYOUT, index=g.INDEX_HASH, fill_seed=SEED, max_batch=BATCH)
    yield eng, init
    eng.close()


@pytest.fixture(scope="module")
def theta06(big_table):
    eng, init = big_table
    txs = g.gen_ycsb(BIG_ROWS, 4 * BATCH, 0.6, 0.9, seed=SEED, dedup=g.DEDUP_RESAMPLE, key_base=0)
    return eng, init, txs


@pytest.mark.parametrize("scheme", g.SCHEMES)
def test_bench_shape_theta06_per_batch_launches(oracle, theta06, scheme):
    eng, init, txs = theta06
    eng.load_txs(txs)
    res = run(eng, init, scheme, BATCH)
    assert res["batches"] == (1 if scheme == "gputx" else 4)
    check(oracle, eng, init, txs, scheme, res, 7)


@pytest.mark.parametrize("scheme", g.QUEUE_SCHEMES)
def test_bench_shape_theta06_device_queue(oracle, theta06, scheme):
    eng, init, txs = theta06
    eng.load_txs(txs)
    res = run(eng, init, scheme, BATCH, flags=g.F_QUEUE, write_seed=8)
    assert res["batches"] == 1
    check(oracle, eng, init, txs, scheme, res, 8)


def test_bench_shape_device_queue_from_host(oracle, theta06):
    """gcc_run_host with the device queue: batch b is admitted when its
    records reach the device, while earlier batches execute."""
    eng, init, txs = theta06
    eng.upload_table(init)
    dg_host = np.zeros(len(txs), dtype=np.uint64)
    res = eng.run_host("tpl_nw", txs, dg_host, warp_density=5, block_size=32, batch_size=BATCH,
                       flags=g.F_COMMIT_LOG | g.F_QUEUE, write_seed=9, spin_limit_ns=SPIN_NS)
    assert np.array_equal(dg_host, eng.digests())
    check(oracle, eng, init, txs, "tpl_nw", res, 9)


@pytest.fixture(scope="module")
def theta099(big_table):
    eng, init = big_table
    txs = g.gen_ycsb(BIG_ROWS, 2 * BATCH, 0.99, 0.9, seed=SEED, dedup=g.DEDUP_RESAMPLE,
                     key_base=0)
    return eng, init, txs


@pytest.mark.parametrize("cap", [0, 512])
@pytest.mark.parametrize("scheme", g.SCHEMES)
def test_bench_table_theta099(oracle, theta099, scheme, cap):
    eng, init, txs = theta099
    eng.load_txs(txs)
    res = run(eng, init, scheme, BATCH, max_active=cap)
    check(oracle, eng, init, txs, scheme, res, 7)
    if scheme in ("tpl_nw", "silo") and cap == 0:
        assert res["aborts"] > 0  # the case is contended


@pytest.mark.parametrize("scheme", ["tpl_nw", "silo", "tictoc", "to"])
def test_bench_table_theta099_device_queue(oracle, theta099, scheme):
    eng, init, txs = theta099
    eng.load_txs(txs)
    res = run(eng, init, scheme, BATCH, flags=g.F_QUEUE, max_active=512)
    check(oracle, eng, init, txs, scheme, res, 7)


def test_queue_rejects_unsupported(theta099):
    eng, _, txs = theta099
    eng.load_txs(txs[:1024])
    for scheme in ("mvcc", "gacco", "gputx", "slow_mvcc"):
        with pytest.raises(g.GccError) as ei:
            eng.run(scheme, batch_size=512, flags=g.F_QUEUE)
        assert ei.value.status == -1
    with pytest.raises(g.GccError) as ei:
        eng.run("tpl_nw", batch_size=512, flags=g.F_QUEUE, write_mode=g.WRITE_ROWCOPY)
    assert ei.value.status == -1
