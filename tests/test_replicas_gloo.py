"""The N>1 path (independent replicas, one per GPU) on CPU: two gloo ranks
combine their measurements the way bench.py does under torchrun — device
time is the max over ranks, committed work the sum — and every rank takes
the same collective steps."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(ws), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from gpu_cc_tb_b200 import replicas
    r, w, local, dist = replicas.init_from_env(backend="gloo", timeout_s=30)
    assert (r, w) == (rank, ws)
    replicas.barrier(dist)
    # replica r: 1M committed in (1 + r) s device time, e2e 2 s + r
    out = replicas.combine(dist, device_seconds=1.0 + r, committed=1_000_000,
                           e2e_seconds=2.0 + r, e2e_transactions=1_000_000)
    q.put((rank, out))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_replicas_combine_max_time_and_sum_work():
    ws, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(ws))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(ws):
        out = res[r]
        assert out["device_s_max"] == 2.0
        assert out["committed"] == 2_000_000
        assert out["value"] == pytest.approx(1_000_000.0)
        assert out["e2e_value"] == pytest.approx(2_000_000 / 3.0)


def test_single_process_needs_no_group():
    from gpu_cc_tb_b200 import replicas
    os.environ.pop("WORLD_SIZE", None)
    r, w, local, dist = replicas.init_from_env()
    assert (r, w, dist) == (0, 1, None)
    out = replicas.combine(None, 2.0, 10, 4.0, 10)
    assert out["value"] == 5.0 and out["e2e_value"] == 2.5
