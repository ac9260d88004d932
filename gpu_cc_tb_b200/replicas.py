"""Multi-GPU runs of the engine: independent replicas, one process per GPU.

The YCSB path does not shard (transactions touch arbitrary Zipf keys of one
table; gCCTB has no cross-partition commit), so N GPUs run N independent
engines over the same workload and nothing crosses between them on the data
path. The process group is used only to line the ranks up and to combine
their measurements: device time is the max over ranks (the job takes as long
as its slowest replica), work is the sum.
"""
from __future__ import annotations

import os
from datetime import timedelta

import torch


def init_from_env(backend: str = "nccl", timeout_s: float = 120.0):
    """(rank, world_size, local_rank, dist or None) from torchrun's env."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws <= 1:
        return 0, 1, 0, None
    import torch.distributed as dist
    rank, local = int(os.environ["RANK"]), int(os.environ.get("LOCAL_RANK", "0"))
    if backend == "nccl":
        torch.cuda.set_device(local)
    dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))
    return rank, ws, local, dist


def _device(dist):
    if dist is not None and dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def reduce_max(dist, v: float) -> float:
    if dist is None:
        return float(v)
    t = torch.tensor([float(v)], dtype=torch.float64, device=_device(dist))
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(dist, v: float) -> float:
    if dist is None:
        return float(v)
    t = torch.tensor([float(v)], dtype=torch.float64, device=_device(dist))
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(dist):
    if dist is not None:
        dist.barrier()
    if torch.cuda.is_available() and (dist is None or dist.get_backend() == "nccl"):
        torch.cuda.synchronize()


def combine(dist, device_seconds: float, committed: int, e2e_seconds: float,
            e2e_transactions: int) -> dict:
    """Whole-job figures of a replica run: committed tx/s over the slowest
    replica's device time, and the same for the end-to-end leg."""
    t_max = reduce_max(dist, device_seconds)
    c_sum = reduce_sum(dist, committed)
    e_max = reduce_max(dist, e2e_seconds)
    e_sum = reduce_sum(dist, e2e_transactions)
    return {"device_s_max": t_max, "committed": c_sum,
            "value": c_sum / t_max if t_max > 0 else 0.0,
            "e2e_s_max": e_max, "e2e_value": e_sum / e_max if e_max > 0 else 0.0}
