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
