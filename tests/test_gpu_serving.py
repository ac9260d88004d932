"""Serving loop on the GPU: variable-length (order-entry) transactions
arriving as a Poisson stream, admitted in batches, run with the learned
scheduler on and off. Checks: every transaction commits, the commit-order
replay of the oracle reproduces the final table and every read digest, the
latency figures are ordered and bounded below by the batch service, and the
variable-length predictor features equal the oracle's bit for bit."""
import numpy as np
import pytest

import gpu_cc_tb_b200 as g
from oracle import predictor as P

pytestmark = pytest.mark.gpu
SPIN = 2_000_000_000


@pytest.fixture(scope="module")
def oe():
    d = g.order_entry_desc(warehouses=4, districts=10, customers=300, items=2000)
    n_tx = 20_000
    off, reqs, kind, lay = g.gen_order_entry(d, n_tx, seed=12)
    eng = g.Engine(lay["rows"], layout=g.LAYOUT_U64X11, index=g.INDEX_DIRECT, fill_seed=0,
                   max_batch=4096)
    eng.oe_fill(d, seed=2)
    init = eng.dump_table()
    eng.load_var_txs(off, reqs)
    yield eng, init, off, reqs
    eng.close()


def test_var_features_bit_exact(oe):
    eng, init, off, reqs = oe
    with g.Scheduler(eng) as sc:
        freq = np.zeros(1 << P.FREQ_BITS, dtype=np.uint32)
        sc.observe_var(0, 0, clear=True)
        for lo in (0, 5000):
            sc.observe_var(lo, 5000)
            freq = P.observe_var(freq, off, reqs, lo, lo + 5000)
        got = sc.features_var(2000, 8000)
        want = P.features_var(off, reqs, 2000, 10000, freq)
        assert (want[:, 65] > 0).any() and want[:, :64].sum(axis=1).max() > 16
        assert np.array_equal(got, want)


@pytest.mark.parametrize("scheme", ["tpl_nw", "silo", "tictoc"])
@pytest.mark.parametrize("mode", [g.SCHED_PLAIN, g.SCHED_LEARNED])
def test_serving_commits_and_replays(oracle, oe, scheme, mode):
    eng, init, off, reqs = oe
    n = len(off) - 1
    with g.Scheduler(eng, mode=mode, probe_rows=512, minibatch=512, min_sched=-1) as sc:
        eng.upload_table(init)
        r = sc.serve(scheme, rate_tps=400_000, seed=3, max_batch=4096, warp_density=5,
                     block_size=8, flags=g.F_COMMIT_LOG | g.F_EXT_OPS | g.F_NO_RESET,
                     write_seed=21, spin_limit_ns=SPIN)
        assert r["committed"] == n
        assert 1 <= r["batches"] <= n and r["admit_cap"] == 4096
        assert 0 < r["lat_p50_us"] <= r["lat_p99_us"] <= r["lat_max_us"]
        assert 300_000 < r["offered_tps"] < 500_000
        recs = sc.batches()
        assert sum(b["committed"] for b in recs) == n
        if mode == g.SCHED_LEARNED:
            assert any(b["probe"] for b in recs)
        table, dg = eng.dump_table(), eng.digests()
        order = oracle.commit_order(eng.commit_log())
        ref_t, ref_dg = oracle.replay_var(init, g.LAYOUT_U64X11, off, reqs, order,
                                          g.WRITE_FIELD, 21, ext_ops=True)
        assert np.array_equal(table, ref_t)
        assert np.array_equal(dg, ref_dg)


def test_serving_admission_cap_from_device_memory(oe):
    eng, init, off, reqs = oe
    with g.Scheduler(eng, mode=g.SCHED_PLAIN) as sc:
        eng.upload_table(init)
        r = sc.serve("tpl_nw", rate_tps=5e7, seed=4, warp_density=5, block_size=32,
                     flags=g.F_EXT_OPS | g.F_NO_RESET, write_seed=1, spin_limit_ns=SPIN)
        assert r["committed"] == len(off) - 1
        # nearly everything arrives before the first batch ends: few, large batches
        assert r["admit_cap"] == len(off) - 1 and r["batches"] <= 8
        with pytest.raises(g.GccError):
            sc.serve("mvcc", rate_tps=1e5, flags=g.F_EXT_OPS)
