"""gcc_run_host: records streamed from host memory batch by batch, digests
streamed back, must give what load + run + read-back gives: the same final
table and digests for the deterministic order (GaccO, GPUTx), and a
commit-order replay that matches for a concurrent scheme."""
import numpy as np
import pytest
import torch

import gpu_cc_tb_b200 as g

pytestmark = pytest.mark.gpu


def _pinned(a):
    t = torch.empty(a.nbytes, dtype=torch.uint8, pin_memory=True)
    v = t.numpy().view(a.dtype)
    v[:] = a
    return t, v


@pytest.mark.parametrize("scheme", ["gacco", "gputx", "tpl_nw", "silo"])
def test_run_host_matches_load_and_run(oracle, scheme):
    rows = 50_000
    txs = g.gen_ycsb(rows, 20_000, 0.8, 0.7, seed=19, dedup=g.DEDUP_RESAMPLE, key_base=0)
    init = oracle.fill_table(rows, g.LAYOUT_U64X11, 6)
    keep, host = _pinned(txs)
    dg_host = np.zeros(len(txs), dtype=np.uint64)
    with g.Engine(rows, layout=g.LAYOUT_U64X11, index=g.INDEX_HASH, fill_seed=6,
                  max_batch=4096) as eng:
        kw = dict(warp_density=5, block_size=16, batch_size=4096, write_seed=3,
                  flags=g.F_COMMIT_LOG)
        r = eng.run_host(scheme, host, dg_host, **kw)
        assert r["committed"] == len(txs) and r["batches"] == (1 if scheme == "gputx" else 5)
        t_host = eng.dump_table()
        assert np.array_equal(dg_host, eng.digests())
        if scheme in ("gacco", "gputx"):
            eng.upload_table(init)
            eng.load_txs(txs)
            eng.run(scheme, **kw)
            assert np.array_equal(t_host, eng.dump_table())
            assert np.array_equal(dg_host, eng.digests())
        else:
            order = oracle.commit_order(eng.commit_log())
            ref_t, ref_dg, _ = oracle.replay(init, g.LAYOUT_U64X11, txs, order, g.WRITE_FIELD, 3)
            assert np.array_equal(t_host, ref_t) and np.array_equal(dg_host, ref_dg)
    del keep
