"""The oracle's extended request ops, pinned by hand-worked cases (the stock
rule's wrap, payments, inserts), and the order-entry generator's prefix
property that the serving bench relies on (the first n transactions of a
stream are the same whatever its length)."""
import numpy as np

import gpu_cc_tb_b200 as g


def _table(rows):
    t = np.zeros((rows, 11), dtype=np.uint64)
    t[:, 0] = np.arange(rows)
    return t


def test_extended_ops_known_answers(oracle):
    t = _table(8)
    t[1, 1:5] = [50, 7, 3, 0]          # stock: quantity 50
    t[2, 1:5] = [12, 0, 0, 0]          # stock: quantity 12 (wraps)
    t[3, 1:4] = [1000, 0, 0]           # customer: balance, ytd, count
    t[4, 1] = 10                       # plain counter
    reqs = np.zeros(6, dtype=g.REQ_DTYPE)
    reqs[0] = (g.op_word(g.OP_STOCK, 0, 5), 1)            # 50 - 5 = 45
    reqs[1] = (g.op_word(g.OP_STOCK, 0, 5 | 0x100), 2)    # 12 - 5 + 91 = 98, remote
    reqs[2] = (g.op_word(g.OP_PAY, 0, 300), 3)
    reqs[3] = (g.op_word(g.OP_ADD, 0, 5), 4)
    reqs[4] = (g.op_word(g.OP_SUB, 0, 20), 4)             # 10 + 5 - 20 = -5 (two's complement)
    reqs[5] = (g.op_word(g.OP_INSERT, 0, 77), 6)
    off = np.array([0, 6], dtype=np.uint32)
    out, dg = oracle.replay_var(t.view(np.uint8).reshape(8, 88), g.LAYOUT_U64X11, off, reqs,
                                None, g.WRITE_FIELD, 9, ext_ops=True)
    o = out.view(np.uint64).reshape(8, 11)
    assert list(o[1, 1:5]) == [45, 12, 4, 0]
    assert list(o[2, 1:5]) == [98, 5, 1, 1]
    assert list(o[3, 1:4]) == [700, 300, 1]
    assert int(o[4, 1].astype(np.int64)) == -5
    assert o[6, 1] == 0 and o[6, 2] == 77 and (o[6, 3:] != 0).all()
    assert dg[0] != 0
    # without ext_ops the same words are plain YCSB field writes
    out2, _ = oracle.replay_var(t.view(np.uint8).reshape(8, 88), g.LAYOUT_U64X11, off, reqs,
                                None, g.WRITE_FIELD, 9, ext_ops=False)
    assert not np.array_equal(out2, out)


def test_malformed_op_is_rejected(oracle):
    t = _table(4)
    reqs = np.zeros(1, dtype=g.REQ_DTYPE)
    reqs[0] = (g.op_word(g.OP_STOCK, 9, 1), 1)            # field 9 + 3 leaves the row
    import pytest
    with pytest.raises(RuntimeError):
        oracle.replay_var(t.view(np.uint8).reshape(4, 88), g.LAYOUT_U64X11,
                          np.array([0, 1], dtype=np.uint32), reqs, None, g.WRITE_FIELD, 1,
                          ext_ops=True)


def test_generator_prefix_property():
    d = g.order_entry_desc(warehouses=8)
    off_a, reqs_a, kind_a, lay_a = g.gen_order_entry(d, 3000, seed=4)
    off_b, reqs_b, kind_b, lay_b = g.gen_order_entry(d, 5000, seed=4)
    assert np.array_equal(off_a, off_b[:3001])
    assert np.array_equal(reqs_a, reqs_b[:int(off_a[-1])])
    assert np.array_equal(kind_a, kind_b[:3000])
    assert lay_a["inserts"] == lay_b["inserts"] and lay_a["rows"] < lay_b["rows"]


import pytest


@pytest.mark.parametrize("scheme", ["tpl_nw", "silo", "tictoc"])
def test_cpu_executors_on_order_entry(oracle, scheme):
    # the multi-threaded CPU executors (the timed CPU baseline of the
    # order-entry workload) are serializable: their commit order replays to
    # the same table and digests
    d = g.order_entry_desc(warehouses=2, districts=4, customers=50, items=500)
    off, reqs, kind, lay = g.gen_order_entry(d, 3000, seed=8)
    init = oracle.fill_table(lay["rows"], g.LAYOUT_U64X11, 5)
    t, dg, log, secs, aborts = oracle.cpu_run_var(scheme, init, g.LAYOUT_U64X11, off, reqs,
                                                  g.WRITE_FIELD, 3, ext_ops=True, threads=4)
    order = oracle.commit_order(log)
    ref_t, ref_dg = oracle.replay_var(init, g.LAYOUT_U64X11, off, reqs, order, g.WRITE_FIELD, 3,
                                      ext_ops=True)
    assert np.array_equal(t, ref_t) and np.array_equal(dg, ref_dg)
    assert secs > 0
