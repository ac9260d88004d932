"""Batched execution of variable-length transactions (4-64 requests) on the
GPU: one launch per batch (the reference's batch loop) and one persistent
kernel draining every batch from a device queue, with CUDA-graph replay and
the per-batch autotuner. Parity bar as everywhere: replaying the committed
transactions in their logged serialization order reproduces the final
table and every read digest bit for bit."""
import numpy as np
import pytest

import gpu_cc_tb_b200 as g

pytestmark = pytest.mark.gpu
SPIN = 2_000_000_000


@pytest.fixture(scope="module")
def var_setup(oracle):
    rows = 200000
    off, reqs = g.gen_ycsb_var(rows, 6000, 0.6, 0.8, min_ops=4, max_ops=64, seed=17)
    init = oracle.fill_table(rows, g.LAYOUT_U64X11, 3)
    eng = g.Engine(rows, layout=g.LAYOUT_U64X11, index=g.INDEX_HASH, fill_seed=3, max_batch=4096)
    eng.load_var_txs(off, reqs)
    yield eng, init, off, reqs
    eng.close()


BATCHES = np.array([0, 500, 2500, 2600, 6000], dtype=np.uint32)  # uneven


def check(oracle, eng, init, off, reqs, seed):
    table = eng.dump_table()
    dg = eng.digests()
    order = oracle.commit_order(eng.commit_log())
    rt, rdg = oracle.replay_var(init, g.LAYOUT_U64X11, off, reqs, order, g.WRITE_FIELD, seed)
    bad = np.nonzero((table != rt).any(axis=1))[0]
    assert len(bad) == 0, f"{len(bad)} rows differ"
    assert np.array_equal(dg, rdg), f"{np.count_nonzero(dg != rdg)} digests differ"


@pytest.mark.parametrize("mode", [g.BATCHES_SEQUENTIAL, g.BATCHES_QUEUE])
@pytest.mark.parametrize("scheme", g.VAR_SCHEMES)
@pytest.mark.parametrize("wd", [5, 3])
def test_batches_parity(oracle, var_setup, scheme, mode, wd):
    eng, init, off, reqs = var_setup
    if mode == g.BATCHES_QUEUE and scheme in ("mvcc", "slow_mvcc"):
        with pytest.raises(g.GccError):
            eng.run_batches(scheme, BATCHES, mode, warp_density=wd, block_size=8)
        return
    eng.upload_table(init)
    res = eng.run_batches(scheme, BATCHES, mode, warp_density=wd, block_size=8,
                          flags=g.F_COMMIT_LOG, write_seed=21, spin_limit_ns=SPIN)
    assert res["committed"] == len(off) - 1
    check(oracle, eng, init, off, reqs, 21)


def test_graph_replay_and_autotune(oracle, var_setup):
    eng, init, off, reqs = var_setup
    seen = set()
    for run in range(8):
        eng.upload_table(init)
        res = eng.run_batches("tictoc", BATCHES, g.BATCHES_SEQUENTIAL, warp_density=5,
                              block_size=32, flags=g.F_COMMIT_LOG | g.F_AUTOTUNE | g.F_GRAPH,
                              write_seed=5, spin_limit_ns=SPIN)
        assert res["committed"] == len(off) - 1
        check(oracle, eng, init, off, reqs, 5)
        wd, bs, ms = eng.batch_stats()
        act = eng.batch_active()
        assert len(wd) == 4 and (ms > 0).all() and (act > 0).all()
        seen.update(zip(wd.tolist(), bs.tolist(), act.tolist()))
    assert len(seen) >= 3  # the tuner explored several configurations
    for run in range(2):
        eng.upload_table(init)
        eng.run_batches("silo", BATCHES, g.BATCHES_QUEUE, warp_density=4, block_size=16,
                        flags=g.F_COMMIT_LOG | g.F_GRAPH, write_seed=6, spin_limit_ns=SPIN)
        check(oracle, eng, init, off, reqs, 6)


def test_batches_reject_bad_arguments(var_setup):
    eng, init, off, reqs = var_setup
    with pytest.raises(g.GccError):
        eng.run_batches("gacco", BATCHES)          # ordered schemes: not batched
    with pytest.raises(g.GccError):
        eng.run_batches("tpl_nw", np.array([0, 10], dtype=np.uint32))  # must cover all txs
    with pytest.raises(g.GccError):
        eng.run_batches("tpl_nw", BATCHES, warp_density=1)


def test_autotuner_batch_size_arms(oracle):
    """The tuner's arms include batch_size (launches of at most 16,384 /
    65,536 transactions inside a batch); a batch cut into launches still
    replays bit-exactly."""
    rows = 200000
    off, reqs = g.gen_ycsb_var(rows, 40000, 0.6, 0.8, min_ops=4, max_ops=32, seed=23)
    init = oracle.fill_table(rows, g.LAYOUT_U64X11, 3)
    boff = np.array([0, 20000, 40000], dtype=np.uint32)
    splits = set()
    with g.Engine(rows, layout=g.LAYOUT_U64X11, index=g.INDEX_HASH, fill_seed=3,
                  max_batch=20000) as eng:
        eng.load_var_txs(off, reqs)
        for run in range(11):
            eng.upload_table(init)
            res = eng.run_batches("tpl_nw", boff, g.BATCHES_SEQUENTIAL, warp_density=5,
                                  block_size=32, flags=g.F_COMMIT_LOG | g.F_AUTOTUNE,
                                  write_seed=9, spin_limit_ns=SPIN)
            assert res["committed"] == len(off) - 1
            check(oracle, eng, init, off, reqs, 9)
            sp = eng.batch_split()
            assert set(sp.tolist()) <= {0, 16384, 65536}
            splits.update(sp.tolist())
            if 16384 in sp.tolist():
                assert res["kernel_launches"] >= 2 * 3  # 2 launches for a 20,000 batch
    assert 16384 in splits or 65536 in splits
