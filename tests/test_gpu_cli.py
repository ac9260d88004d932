"""The CLI drop-ins on the GPU: gen_ycsb writes the reference's record format,
test_ycsb runs it with the reference's positional arguments, prints the result
block, appends the 15-column line to <dataset>.txt, and with debug_flag=1
checks serializability by re-executing the committed transactions in their
serialization order (GOOD/BAD, the role of src/runtime.cu:129-158)."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

import gpu_cc_tb_b200 as g

pytestmark = pytest.mark.gpu
BIN = Path(g.__file__).resolve().parent / "bin"


@pytest.fixture(scope="module")
def dataset(tmp_path_factory):
    d = tmp_path_factory.mktemp("cli")
    path = d / "ycsb.txs"
    out = subprocess.run([str(BIN / "gen_ycsb"), "4096", "8192", "0.8", "0.5", str(path)],
                         capture_output=True, text=True, check=True)
    assert "GEN OK" in out.stdout
    recs = np.frombuffer(path.read_bytes(), dtype=g.TX_DTYPE)
    assert len(recs) == 8192 and recs["request_cnt"].max() <= 16
    return path


@pytest.mark.parametrize("scheme", ["tpl_nw", "tpl_wd", "to", "mvcc", "silo", "tictoc", "gacco",
                                    "gputx", "slow_tpl_nw", "slow_silo", "slowto", "slowmvcc"])
def test_test_ycsb_debug_check_is_good(dataset, scheme):
    out = subprocess.run([str(BIN / "test_ycsb"), str(dataset), "4096", "8192", scheme, "5", "8",
                          "2048", "1"], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    lines = out.stdout.splitlines()
    assert lines[0] == f"TRY {scheme},5,8,2048"
    assert lines[-1] == "GOOD", out.stdout
    assert any(l.startswith("through ") for l in lines)
    csv = (Path(str(dataset) + ".txt")).read_text().splitlines()
    last = csv[-1].split(",")
    assert len(last) == 15 and last[0] == scheme


def test_test_ycsb_rejects_reference_knob_limits(dataset):
    for wd, bs in (("6", "4"), ("5", "33")):
        out = subprocess.run([str(BIN / "test_ycsb"), str(dataset), "4096", "16", "tpl_nw", wd, bs,
                              "16", "0"], capture_output=True, text=True)
        assert out.returncode == 255  # `return -1` of benchmark_cpu/ycsb.cu:97-98


def test_run_checked_api():
    rows = 2048
    txs = g.gen_ycsb(rows, 4096, 0.9, 0.6, seed=9, dedup=g.DEDUP_RESAMPLE, key_base=0)
    with g.Engine(rows, layout=g.LAYOUT_U64X11, index=g.INDEX_HASH, fill_seed=3,
                  max_batch=1024) as eng:
        eng.load_txs(txs)
        for scheme in ("tpl_nw", "silo", "tictoc", "to", "gacco", "gputx"):
            for mode in (g.WRITE_FIELD, g.WRITE_ROWCOPY):
                res, ok = eng.run_checked(scheme, warp_density=4, block_size=8, batch_size=1024,
                                          write_mode=mode)
                assert ok, (scheme, mode)
                assert res["committed"] == len(txs)


@pytest.mark.parametrize("scheme", ["tpl_nw", "tictoc", "gacco"])
def test_test_ycsb_result_files(oracle, dataset, scheme, tmp_path):
    # the reference's setup (104-byte rows, sorted index, whole-row copies)
    # with every result file written; the files reproduce the oracle's
    # serial replay in the logged order
    outs = {k: tmp_path / f"{k}.bin" for k in ("table", "digests", "commit_log", "aborts", "read_log")}
    args = [str(BIN / "test_ycsb"), str(dataset), "4096", "8192", scheme, "5", "8", "2048", "0"]
    args += [f"{k}_out={v}" for k, v in outs.items()]
    out = subprocess.run(args, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    txs = np.frombuffer(dataset.read_bytes(), dtype=g.TX_DTYPE)
    layout = g.LAYOUT_REF104
    table = np.frombuffer(outs["table"].read_bytes(), dtype=np.uint8).reshape(4096, 104)
    dg = np.frombuffer(outs["digests"].read_bytes(), dtype=np.uint64)
    log = np.frombuffer(outs["commit_log"].read_bytes(), dtype=np.uint64).reshape(-1, 2)
    aborts = np.frombuffer(outs["aborts"].read_bytes(), dtype=np.uint32)
    rl = np.frombuffer(outs["read_log"].read_bytes(), dtype=np.uint8).reshape(8192, 16, 112)
    assert len(dg) == len(log) == len(aborts) == 8192
    order = np.arange(8192) if scheme == "gacco" else oracle.commit_order(log)
    init = oracle.fill_table(4096, layout, 0)
    ref_t, ref_dg, ref_rl = oracle.replay(init, layout, txs, order, g.WRITE_ROWCOPY, 1,
                                          read_log=True)
    assert np.array_equal(table, ref_t)
    assert np.array_equal(dg, ref_dg)
    for t in range(0, 8192, 97):
        for i in range(int(txs[t]["request_cnt"])):
            if txs[t]["requests"][i]["read"]:
                assert np.array_equal(rl[t, i, :104], ref_rl[t, i, :104]), (t, i)
    if scheme == "gacco":
        assert not aborts.any()
