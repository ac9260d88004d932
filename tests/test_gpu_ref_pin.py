"""Pins the deterministic schemes to the reference's own output on the GPU.

The reference's test_ycsb, compiled from its sources into oracle/_ref/
(`make -C oracle ref REF=<reference dir>`), runs in its dump variant: rows
and the kernel's `Item item` start at zero instead of uninitialised memory
and the final table is written out after cc->Sync() (the three edits are
listed in oracle/Makefile). Its final table must equal the engine's byte for
byte on the same records, in the reference's own format: 104-byte Item rows
(id = row, fields zero), the sorted-array index, keys in [1, rows-1],
repeated keys dropped, and writes that copy the transaction's last read row
over the whole target row (benchmark/ycsb.cu:57-98).

  * gacco: per-object hand-off in transaction order inside each batch
    (include/gacco.cuh:156-175). The reference waits on lower transactions
    without a bound, so every batch here fits in one wave of resident CTAs
    (batch x 32 threads <= 148 x 1,024). One dataset comes from the
    reference's own gen_ycsb.
  * gputx: rank-ordered execution (src/gputx.cu:5-38). The reference runs a
    rank in one launch, so transactions of equal rank that conflict race, and
    its rank pass reads the last accessed row's list end past its scanned
    offsets; the datasets are seeds on which neither happens (checked with
    oracle_py.gputx_rank_hazards), with up to 7 ranks.

With 104-byte row copies the final table records where every written row's
bytes came from, so the comparison checks the order of every conflicting
access pair.
"""
import subprocess

import numpy as np
import pytest

import gpu_cc_tb_b200 as g
from oracle import oracle_py as o
from oracle import ref_gpu

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def need_reference():
    if not ref_gpu.available(dump=True):
        pytest.skip("the reference build is missing (make -C oracle ref REF=<reference dir>)")


def engine_table(txs, rows, scheme, batch):
    with g.Engine(rows, layout=g.LAYOUT_REF104, index=g.INDEX_SORTED, fill_seed=0,
                  max_batch=batch) as eng:
        init = eng.dump_table()
        eng.load_txs(txs)
        res = eng.run(scheme, warp_density=5, block_size=32, batch_size=batch,
                      write_mode=g.WRITE_ROWCOPY, spin_limit_ns=4_000_000_000)
        assert res["committed"] == len(txs)
        return init, eng.dump_table()


def reference_table(tmp_path, txs, rows, scheme, batch):
    ds = tmp_path / f"{scheme}.txs"
    ds.write_bytes(txs.tobytes())
    out = tmp_path / f"{scheme}.table"
    ref_gpu.run(ds, rows, len(txs), scheme, 5, 32, batch, dump_table=out, timeout=600)
    return np.frombuffer(out.read_bytes(), dtype=np.uint8).reshape(rows, 104)


def compare(init, mine, ref):
    assert (init[:, 4:] == 0).all() and (ref != init).any(axis=1).sum() > 0
    bad = np.nonzero((mine != ref).any(axis=1))[0]
    assert len(bad) == 0, f"{len(bad)} rows differ from the reference, e.g. {bad[:8]}"


@pytest.mark.parametrize("rows,n_tx,theta,r,batch,seed", [
    (65536, 32768, 0.6, 0.5, 4096, 7),
    (16384, 16384, 0.9, 0.8, 2048, 3),
])
def test_gacco_equals_reference(tmp_path, rows, n_tx, theta, r, batch, seed):
    assert batch * 32 <= ref_gpu.ONE_WAVE_THREADS
    txs = o.gen_ycsb(rows, n_tx, theta, r, seed, 0, 1)  # dedup drop, keys 1..rows-1
    ref = reference_table(tmp_path, txs, rows, "gacco", batch)
    init, mine = engine_table(txs, rows, "gacco", batch)
    compare(init, mine, ref)


def test_gacco_equals_reference_on_its_own_dataset(tmp_path):
    gen = ref_gpu.REF / "gen_ycsb"
    if not gen.exists():
        pytest.skip("the reference's gen_ycsb is missing")
    rows, n_tx, batch = 65536, 16384, 4096
    ds = tmp_path / "ref.txs"
    subprocess.run([str(gen), str(rows), str(n_tx), "0.7", "0.6", str(ds)], check=True,
                   capture_output=True, cwd=tmp_path)
    txs = np.frombuffer(ds.read_bytes(), dtype=o.TX_DTYPE).copy()
    assert len(txs) == n_tx
    ref = reference_table(tmp_path, txs, rows, "gacco", batch)
    init, mine = engine_table(txs, rows, "gacco", batch)
    compare(init, mine, ref)


@pytest.mark.parametrize("rows,n_tx,theta,r,seed", [
    (1048576, 256, 0.6, 0.9, 23),
    (1048576, 256, 0.7, 0.9, 11),
    (1048576, 512, 0.6, 0.9, 11),
    (262144, 256, 0.6, 0.9, 23),
])
def test_gputx_equals_reference_without_rank_races(tmp_path, rows, n_tx, theta, r, seed):
    txs = o.gen_ycsb(rows, n_tx, theta, r, seed, 0, 1)
    same_rank, last = o.gputx_rank_hazards(txs, rows)
    assert same_rank == 0 and last == 1
    _, _, max_rank = o.gputx_order(txs, rows)
    assert max_rank >= 4
    ref = reference_table(tmp_path, txs, rows, "gputx", n_tx)
    init, mine = engine_table(txs, rows, "gputx", n_tx)
    compare(init, mine, ref)
