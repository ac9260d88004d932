"""Order-entry workload: the generator's structure on the CPU, and on the GPU
every scheme that supports extended ops against the oracle's serial replay in
the logged commit order (final table and every read digest bit for bit),
plus the workload's integer invariants (money and counters conserve)."""
import numpy as np
import pytest

import gpu_cc_tb_b200 as g

SPIN = 2_000_000_000


def small_desc():
    return g.order_entry_desc(warehouses=2, districts=10, customers=300, items=2000)


def test_generator_structure():
    d = g.order_entry_desc()
    off, reqs, kind, lay = g.gen_order_entry(d, 50_000, seed=9)
    n = np.diff(off).astype(np.int64)
    assert set(np.unique(kind)) == {1, 2}
    assert 0.45 < (kind == 1).mean() < 0.55
    assert (n[kind == 2] == 4).all()
    lines = (n[kind == 1] - 4) // 3
    assert ((n[kind == 1] - 4) % 3 == 0).all() and lines.min() == 5 and lines.max() == 15
    assert lay["rows"] == lay["inserts"] + int((kind == 2).sum() + (lines + 1).sum())
    keys, ops = reqs["key"].astype(np.int64), reqs["read"]
    for t in range(0, 50_000, 499):
        k = keys[off[t]:off[t + 1]]
        assert (np.diff(k) > 0).all()            # distinct, ascending rows
    assert keys.max() < lay["rows"]
    # every insert slot is used exactly once
    ins = keys[(ops < 0) & (((ops.view(np.uint32) >> 28) & 7) == g.OP_INSERT)]
    assert np.array_equal(np.sort(ins), np.arange(lay["inserts"], lay["rows"]))
    # stock rows of new-orders: NURand(8191) skews items
    st = keys[(ops < 0) & (((ops.view(np.uint32) >> 28) & 7) == g.OP_STOCK)] - lay["stock"]
    item = st % d.items
    assert np.bincount(item, minlength=d.items).max() > 5 * len(item) / d.items
    # determinism
    off2, reqs2, _, _ = g.gen_order_entry(d, 50_000, seed=9, threads=3)
    assert np.array_equal(off, off2) and np.array_equal(reqs, reqs2)


@pytest.mark.gpu
@pytest.mark.parametrize("scheme", ["tpl_nw", "tpl_wd", "to", "silo", "tictoc"])
def test_order_entry_parity(oracle, scheme):
    d = small_desc()
    n_tx = 6000
    off, reqs, kind, lay = g.gen_order_entry(d, n_tx, seed=5)
    boff = np.array([0, 1000, 3000, 6000], dtype=np.uint32)
    with g.Engine(lay["rows"], layout=g.LAYOUT_U64X11, index=g.INDEX_DIRECT, fill_seed=0,
                  max_batch=4096) as eng:
        eng.oe_fill(d, seed=3)
        init = eng.dump_table()
        eng.load_var_txs(off, reqs)
        for mode in (g.BATCHES_SEQUENTIAL, g.BATCHES_QUEUE):
            eng.upload_table(init)
            r = eng.run_batches(scheme, boff, mode, warp_density=5, block_size=8,
                                flags=g.F_COMMIT_LOG | g.F_EXT_OPS, write_seed=17,
                                spin_limit_ns=SPIN)
            assert r["committed"] == n_tx
            table, dg = eng.dump_table(), eng.digests()
            order = oracle.commit_order(eng.commit_log())
            ref_t, ref_dg = oracle.replay_var(init, g.LAYOUT_U64X11, off, reqs, order,
                                              g.WRITE_FIELD, 17, ext_ops=True)
            assert np.array_equal(table, ref_t)
            assert np.array_equal(dg, ref_dg)
    # integer invariants of the final table
    t = table.view(np.uint64).reshape(lay["rows"], 11)
    W, D, C = d.warehouses, d.districts, d.customers
    pay = reqs["read"][(reqs["read"] < 0) & (((reqs["read"].view(np.uint32) >> 28) & 7) == g.OP_PAY)]
    paid = int((pay.view(np.uint32) & 0xFFFFFF).sum())
    it = init.view(np.uint64).reshape(lay["rows"], 11)
    assert int(t[:W, 1].sum() - it[:W, 1].sum()) == paid
    assert int(t[W:W + W * D, 1].sum() - it[W:W + W * D, 1].sum()) == paid
    assert int(t[W:W + W * D, 3].sum() - it[W:W + W * D, 3].sum()) == int((kind == 1).sum())
    cust = slice(lay["customer"], lay["item"])
    assert int((it[cust, 1] - t[cust, 1]).astype(np.int64).sum()) == paid
    lines = int(((np.diff(off)[kind == 1] - 4) // 3).sum())
    stock = slice(lay["stock"], lay["inserts"])
    assert int(t[stock, 3].sum()) == lines


@pytest.mark.gpu
def test_ext_ops_rejected_where_unsupported():
    d = small_desc()
    off, reqs, kind, lay = g.gen_order_entry(d, 100, seed=1)
    with g.Engine(lay["rows"], layout=g.LAYOUT_U64X11, index=g.INDEX_DIRECT, fill_seed=0,
                  max_batch=128) as eng:
        eng.oe_fill(d)
        eng.load_var_txs(off, reqs)
        boff = np.array([0, 100], dtype=np.uint32)
        with pytest.raises(g.GccError):
            eng.run_batches("mvcc", boff, g.BATCHES_SEQUENTIAL, flags=g.F_EXT_OPS)
        # a malformed op word (field out of range) ends the run with EFORMAT
        bad = reqs.copy()
        bad["read"][0] = g.op_word(g.OP_STOCK, 9, 1)
        eng.load_var_txs(off, bad)
        with pytest.raises(g.GccError) as ex:
            eng.run_batches("tpl_nw", boff, g.BATCHES_SEQUENTIAL, flags=g.F_EXT_OPS,
                            spin_limit_ns=SPIN)
        assert ex.value.status == -5
