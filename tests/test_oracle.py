"""The CPU oracle checked on its own: known-answer cases worked by hand from
the reference's algorithms, the committed golden fixtures, and consistency
between its serial replay and its multi-threaded executors."""
import json
from pathlib import Path

import numpy as np
import pytest

import gpu_cc_tb_b200 as g

GOLDEN = Path(__file__).resolve().parent / "golden"


def make_txs(spec):
    """spec: list of transactions, each a list of (read, key)."""
    a = np.zeros(len(spec), dtype=g.TX_DTYPE)
    for t, ops in enumerate(spec):
        a[t]["request_cnt"] = len(ops)
        for i, (r, k) in enumerate(ops):
            a[t]["requests"][i] = (r, k)
    return a


def test_gputx_rank_known_answers(oracle):
    # Object lists in tx order (src/gputx.cu:17-27): rank grows after any
    # pair that is not read/read.
    #  row 1: T0 r, T1 r, T2 w, T3 r  -> ranks 0, 0, 1, 2
    #  row 2: T1 w, T3 w              -> ranks 0, 1
    #  row 3: T0 w, T4 r              -> ranks 0, 1
    txs = make_txs([[(1, 1), (0, 3)], [(1, 1), (0, 2)], [(0, 1)], [(1, 1), (0, 2)], [(1, 3)]])
    ranks, order, mx = oracle.gputx_order(txs, 8)
    assert ranks.tolist() == [0, 0, 1, 2, 1]
    assert order.tolist() == [0, 1, 2, 4, 3]   # (rank, tx)
    assert mx == 2


def test_gputx_single_pass_rank_allows_same_rank_conflict(oracle):
    # y(2): T0 w, T1 r -> T0 0, T1 1 ; x(1): T1 w, T2 r -> T1 0, T2 1.
    # One pass of max gives T1 and T2 the same rank although T2 reads what
    # T1 writes; the engine orders them by tx index inside the rank.
    txs = make_txs([[(0, 2)], [(0, 1), (1, 2)], [(1, 1)]])
    ranks, order, mx = oracle.gputx_order(txs, 4)
    assert ranks.tolist() == [0, 1, 1]
    assert order.tolist() == [0, 1, 2]
    assert mx == 1


def test_replay_semantics_field_and_rowcopy(oracle):
    layout = g.LAYOUT_U64X11
    init = oracle.fill_table(8, layout, 3)
    words = init.view("<u8").reshape(8, 11)
    assert (words[:, 0] == np.arange(8)).all()
    txs = make_txs([[(1, 2), (0, 5)], [(0, 2)], [(1, 5), (1, 6), (0, 7)]])
    # rowcopy: T0 copies row 2 over row 5; T1 writes zeros (no read before);
    # T2 reads rows 5 (= old row 2) and 6, then copies row 6 over row 7.
    t, dg, rl = oracle.replay(init, layout, txs, [0, 1, 2], g.WRITE_ROWCOPY, 0, read_log=True)
    tw = t.view("<u8").reshape(8, 11)
    assert (tw[5] == words[2]).all()
    assert (tw[2] == 0).all()
    assert (tw[7] == words[6]).all()
    assert np.array_equal(rl[2, 0, :88], init[2])
    # digest is a sum of per-word terms: equal for equal reads at equal ops
    assert dg[0] != 0 and dg[1] == 0
    # field writes touch exactly one word of the row
    t2, _, _ = oracle.replay(init, layout, txs, [0, 1, 2], g.WRITE_FIELD, 42)
    diff = (t2.view("<u8").reshape(8, 11) != words)
    assert diff[5].sum() == 1 and diff[2].sum() == 1 and diff[7].sum() == 1
    assert diff[:, 0].sum() == 0


def test_replay_rejects_missing_keys(oracle):
    init = oracle.fill_table(4, 0, 1)
    with pytest.raises(RuntimeError):
        oracle.replay(init, 0, make_txs([[(1, 9)]]), [0], 0, 0)


def test_conflict_checker(oracle):
    E = oracle.EVENT_DTYPE
    # T0 r x, T1 w x, T1 commit, T0 w y? -> T1 depends on T0 (write after
    # T0's active read); T0 then reads y written by active T1 -> cycle.
    ev = np.array([(0, 1, 0, 0, 1), (1, 1, 1, 0, 2), (1, 2, 1, 0, 3), (0, 2, 0, 0, 4),
                   (0, 0, 2, 0, 5), (1, 0, 2, 0, 6)], dtype=E)
    assert not oracle.conflict_acyclic(ev, 2)
    ok = np.array([(0, 1, 0, 0, 1), (0, 0, 2, 0, 2), (1, 1, 1, 0, 3), (1, 0, 2, 0, 4)], dtype=E)
    assert oracle.conflict_acyclic(ok, 2)


@pytest.mark.parametrize("scheme", ["tpl_nw", "silo", "tictoc"])
@pytest.mark.parametrize("write_mode", [g.WRITE_FIELD, g.WRITE_ROWCOPY])
def test_cpu_executors_replay_to_same_state(oracle, scheme, write_mode):
    rows, layout = 300, g.LAYOUT_U64X11
    txs = g.gen_ycsb(rows, 3000, 0.9, 0.6, seed=4, dedup=g.DEDUP_RESAMPLE, key_base=0)
    init = oracle.fill_table(rows, layout, 8)
    t, dg, log, secs, aborts = oracle.cpu_run(scheme, init, layout, txs, write_mode, 17,
                                              threads=8)
    order = oracle.commit_order(log)
    rt, rdg, _ = oracle.replay(init, layout, txs, order, write_mode, 17)
    assert np.array_equal(t, rt) and np.array_equal(dg, rdg)


def test_golden_fixtures(oracle):
    meta = json.loads((GOLDEN / "fixtures.json").read_text())
    for case in meta["cases"]:
        txs = np.frombuffer((GOLDEN / case["txs"]).read_bytes(), dtype=g.TX_DTYPE)
        assert len(txs) == case["n_tx"]
        regen = g.gen_ycsb(case["rows"], case["n_tx"], case["theta"], case["read_ratio"],
                           seed=case["seed"], dedup=case["dedup"], key_base=case["key_base"])
        assert np.array_equal(regen.view(np.uint8), txs.view(np.uint8)), case["name"]
        init = oracle.fill_table(case["rows"], case["layout"], case["fill_seed"])
        if case["order"] == "gputx":
            ranks, order, mx = oracle.gputx_order(txs, case["rows"])
            assert mx == case["max_rank"]
            assert ranks.tolist() == json.loads((GOLDEN / case["ranks"]).read_text())
        else:
            order = np.arange(case["n_tx"])
        t, dg, _ = oracle.replay(init, case["layout"], txs, order, case["write_mode"],
                                 case["write_seed"])
        import hashlib
        assert hashlib.sha256(t.tobytes()).hexdigest() == case["table_sha256"], case["name"]
        assert hashlib.sha256(dg.tobytes()).hexdigest() == case["digests_sha256"], case["name"]


@pytest.mark.parametrize("args", [(100_000, 4000, 0.6, 0.9, 141919810, 1, 0),
                                  (4096, 3000, 0.99, 0.5, 5, 0, 1),
                                  (1_000_000, 2000, 0.1, 1.0, 7, 0, 1)])
def test_oracle_generator_equals_engine_generator(oracle, args):
    """The bench's reference arms take their records from the oracle's
    generator and the engine's arm from its own: they must be the same."""
    rows, n, theta, r, seed, dedup, kb = args
    a = g.gen_ycsb(rows, n, theta, r, seed=seed, dedup=dedup, key_base=kb)
    b = oracle.gen_ycsb(rows, n, theta, r, seed, dedup, kb)
    assert np.array_equal(a.view(np.uint8), b.view(np.uint8))


def test_oracle_write_formulas_match_replay(oracle):
    """write_field / write_value (Python) against the C replay."""
    rows, layout = 8, g.LAYOUT_U64X11
    txs = np.zeros(3, dtype=g.TX_DTYPE)
    for t in range(3):
        txs[t]["request_cnt"] = 2
        txs[t]["requests"][0] = (0, t + 1)
        txs[t]["requests"][1] = (0, t + 4)
    init = oracle.fill_table(rows, layout, 0)
    t_out, _, _ = oracle.replay(init, layout, txs, np.arange(3, dtype=np.uint32), g.WRITE_FIELD, 77)
    w = t_out.view(np.uint64).reshape(rows, 11)
    for t in range(3):
        for i, row in enumerate((t + 1, t + 4)):
            f = oracle.write_field(77, t, i)
            assert int(w[row, 1 + f]) == oracle.write_value(77, t, i)


def test_gputx_rank_hazards_known_answer(oracle):
    """Two transactions that write the same row get ranks 0 and 1 (no
    hazard); adding a third that makes a same-rank write pair is one."""
    rows = 16
    txs = np.zeros(2, dtype=g.TX_DTYPE)
    txs[0]["request_cnt"] = 1
    txs[0]["requests"][0] = (0, 3)
    txs[1]["request_cnt"] = 2
    txs[1]["requests"][0] = (0, 3)
    txs[1]["requests"][1] = (1, 9)
    assert oracle.gputx_rank_hazards(txs, rows) == (0, 1)
    # tx2 reads row 5 (rank 0 there) and writes row 9 after tx1's read
    # (rank 1 there): rank 1 equals tx1's, and both touch row 9 with a write
    t3 = np.zeros(3, dtype=g.TX_DTYPE)
    t3[:2] = txs
    t3[2]["request_cnt"] = 2
    t3[2]["requests"][0] = (1, 5)
    t3[2]["requests"][1] = (0, 9)
    sr, last = oracle.gputx_rank_hazards(t3, rows)
    assert sr == 1 and last == 2
