"""Pin the dataset generator against the reference's own gen_ycsb, built
from its sources into oracle/_ref/ (`make -C oracle ref`; host-only code).

The reference draws from rand() shared by 256 threads, so its datasets are
not reproducible (generation/gen_ycsb.cu:13,44-50); the pin is therefore on
the record format and on the distributions: request counts after dropping
repeated keys, read fraction, key range, per-record key order, and the
Zipfian key frequencies (two-sample KS test)."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

import gpu_cc_tb_b200 as g

REF_GEN = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "gen_ycsb"


@pytest.fixture(scope="module")
def ref_bin():
    if not REF_GEN.exists():
        pytest.skip("oracle/_ref/gen_ycsb not built (make -C oracle ref)")
    return REF_GEN


@pytest.mark.parametrize("rows,n_tx,theta,r", [(2000, 20000, 0.8, 0.9), (50000, 20000, 0.6, 0.5)])
def test_generator_matches_reference_distribution(ref_bin, tmp_path, rows, n_tx, theta, r):
    from scipy import stats

    out = tmp_path / "ref.txs"
    subprocess.run([str(ref_bin), str(rows), str(n_tx), str(theta), str(r), str(out)], check=True,
                   capture_output=True, cwd=tmp_path)
    ref = np.frombuffer(out.read_bytes(), dtype=g.TX_DTYPE)
    assert len(ref) == n_tx
    mine = g.gen_ycsb(rows, n_tx, theta, r, seed=141919810, dedup=g.DEDUP_DROP, key_base=1)

    def flat(a):
        cnt = a["request_cnt"].astype(np.int64)
        mask = np.arange(16)[None, :] < cnt[:, None]
        return cnt, a["requests"]["key"][mask], a["requests"]["read"][mask]

    rc, rk, rr = flat(ref)
    mc, mk, mr = flat(mine)
    # format: counts <= 16, keys distinct + ascending in each record, range
    assert rc.max() <= 16 and mc.max() <= 16
    for a in (ref, mine):
        k = a["requests"]["key"].astype(np.int64)
        cnt = a["request_cnt"].astype(np.int64)
        for t in range(0, len(a), 97):
            assert (np.diff(k[t, : cnt[t]]) > 0).all()
    assert rk.min() >= 1 and rk.max() <= rows - 1
    assert mk.min() >= 1 and mk.max() <= rows - 1
    # distributions
    assert abs(rc.mean() - mc.mean()) < 0.05, (rc.mean(), mc.mean())
    assert abs(rr.mean() - mr.mean()) < 0.01, (rr.mean(), mr.mean())
    ks = stats.ks_2samp(rk, mk)
    assert ks.pvalue > 1e-4, ks
    # the hottest keys are the low ranks in both
    top_ref = np.bincount(rk, minlength=rows)[:5] / len(rk)
    top_mine = np.bincount(mk, minlength=rows)[:5] / len(mk)
    assert np.allclose(top_ref, top_mine, atol=0.01), (top_ref, top_mine)
