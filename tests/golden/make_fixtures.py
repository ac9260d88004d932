"""Regenerate the golden fixtures of tests/test_oracle.py.

Each case is a small dataset from the engine's generator (gen_ycsb format,
136-byte records) plus the SHA-256 of the oracle's serial result (final
table bytes, per-tx read digests) and, for the GPUTx case, the per-tx ranks
of the reference's rank function. Run from the repository root:
    python tests/golden/make_fixtures.py
"""
import hashlib
import json
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))

import numpy as np  # noqa: E402

import gpu_cc_tb_b200 as g  # noqa: E402
from oracle import oracle_py as o  # noqa: E402

CASES = [
    dict(name="u64_field_txorder", rows=512, n_tx=256, theta=0.8, read_ratio=0.7, seed=31,
         dedup=g.DEDUP_RESAMPLE, key_base=0, layout=g.LAYOUT_U64X11, fill_seed=141919810,
         write_mode=g.WRITE_FIELD, write_seed=7, order="tx"),
    dict(name="ref104_rowcopy_txorder", rows=300, n_tx=200, theta=0.6, read_ratio=0.5, seed=32,
         dedup=g.DEDUP_DROP, key_base=1, layout=g.LAYOUT_REF104, fill_seed=0,
         write_mode=g.WRITE_ROWCOPY, write_seed=0, order="tx"),
    dict(name="u64_field_gputx", rows=128, n_tx=300, theta=0.9, read_ratio=0.6, seed=33,
         dedup=g.DEDUP_RESAMPLE, key_base=0, layout=g.LAYOUT_U64X11, fill_seed=5,
         write_mode=g.WRITE_FIELD, write_seed=3, order="gputx"),
]


def main():
    out = []
    for c in CASES:
        txs = g.gen_ycsb(c["rows"], c["n_tx"], c["theta"], c["read_ratio"], seed=c["seed"],
                         dedup=c["dedup"], key_base=c["key_base"])
        fn = f"{c['name']}.txs"
        (HERE / fn).write_bytes(txs.tobytes())
        init = o.fill_table(c["rows"], c["layout"], c["fill_seed"])
        case = dict(c, txs=fn)
        if c["order"] == "gputx":
            ranks, order, mx = o.gputx_order(txs, c["rows"])
            rf = f"{c['name']}.ranks.json"
            (HERE / rf).write_text(json.dumps(ranks.tolist()))
            case.update(ranks=rf, max_rank=mx)
        else:
            order = np.arange(c["n_tx"])
        t, dg, _ = o.replay(init, c["layout"], txs, order, c["write_mode"], c["write_seed"])
        case["table_sha256"] = hashlib.sha256(t.tobytes()).hexdigest()
        case["digests_sha256"] = hashlib.sha256(dg.tobytes()).hexdigest()
        out.append(case)
    (HERE / "fixtures.json").write_text(json.dumps({"cases": out}, indent=1) + "\n")


if __name__ == "__main__":
    main()
