"""Benchmark: committed YCSB transactions per second on B200.

Workload (one point of the plain-YCSB scheme sweep): 10,485,760 rows of
uint64 key + 10 uint64 fields (88 B, stored at a 96 B stride), 1,048,576
transactions of 16 requests, Zipfian keys (theta), reads with probability
`read_ratio`, a write stores a fresh uint64 into one uniformly chosen field,
batch_size 65,536, warp_density 5, block_size 32. A step is one pass of the
engine over all transactions (metadata reset + ordering passes + transaction
kernels, gCCTB's tot_time definition, benchmark_cpu/ycsb.cu:249-291).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--scheme tpl_nw]
  python bench.py --impl reference ...   # the CPU executor on the host cores
  python bench.py --workload batched ...  # 64 uneven batches, 4-64 requests/tx
  python bench.py --workload learned ...  # drifting contention, learned scheduling
  python bench.py --workload serving ...  # order-entry arrivals, p50/p99 latency

The batched workload: 64 consecutive batches with log-uniform sizes in
[4096, 262144] transactions of 4-64 requests (uniform), theta 0.8, read ratio
0.9, on the same table; the device-queue executor (one persistent kernel,
CUDA graph, autotuned warp_density/block_size/transactions in flight) against
the same batches launched one by one with plain kernels.

The learned-scheduling workload: 256 batches of 65,536 transactions of 16
requests on the same table, Zipf theta drifting linearly from 0.5 to 0.99
and read ratio from 0.9 to 0.5 across the batches; the learned scheduler
(BF16 MLP contention predictor, deferral into capped sub-batches, measured
policy) against plain ordering on identical batches through the same driver.

The serving workload: integer order-entry transactions (64 warehouses x 10
districts x 3,000 customers, 100,000 items and stock rows per warehouse;
50% new-order with 5-15 NURand(8191) lines, 1% remote lines; 50% payment,
15% remote customers, 1-5000 cents) arriving as a Poisson process at 10% to
120% of the measured peak rate; batches admitted by free device memory,
table and CC state resident; p50/p99 arrival-to-commit latency and commits/s
with the learned scheduler on and off.

Multi-GPU runs are independent replicas (the path does not shard): every
rank runs the whole workload on its own GPU; value = all ranks' committed
transactions / max over ranks of the device time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

HBM_FALLBACK_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--scheme", default="tpl_nw")
    ap.add_argument("--theta", type=float, default=None,
                    help="Zipf theta (default 0.6 plain, 0.8 batched)")
    ap.add_argument("--read-ratio", type=float, default=0.9)
    ap.add_argument("--rows", type=int, default=10_485_760)
    ap.add_argument("--txs", type=int, default=1_048_576)
    ap.add_argument("--batch", type=int, default=65_536)
    ap.add_argument("--wd", type=int, default=5)
    ap.add_argument("--bs", type=int, default=32)
    ap.add_argument("--index", default="hash", choices=["hash", "sorted", "direct"])
    ap.add_argument("--no-reset", action="store_true")
    ap.add_argument("--no-queue", action="store_true",
                    help="plain workload: one launch per batch (the reference's loop) "
                         "instead of the device queue")
    ap.add_argument("--cpu-threads", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-learned", action="store_true",
                    help="skip the learned-vs-plain comparison at theta 0.99")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip timing the reference's own GPU build (oracle/_ref)")
    ap.add_argument("--sweep", default="tpl_wd,to,mvcc,silo,tictoc,gacco,gputx",
                    help="comma list of extra schemes timed once on the same workload "
                         "('' for none)")
    ap.add_argument("--workload", default="plain",
                    choices=["plain", "batched", "learned", "serving", "sweep"],
                    help="plain: 1,048,576 x 16-request transactions in 65,536 batches; "
                         "batched: 64 uneven batches of 4-64-request transactions; "
                         "learned: 256 drifting-contention batches, learned scheduling")
    ap.add_argument("--sweep-txs", type=int, default=262_144,
                    help="transactions per point of the sweep workload's scheme grid")
    ap.add_argument("--sweep-grid", type=int, default=1,
                    help="sweep workload: 0 skips the scheme x theta x read-ratio grid")
    ap.add_argument("--ref-points", default="ro,mc,hc,t9",
                    help="sweep workload: the reference's dataset points to run")
    ap.add_argument("--batches", type=int, default=None,
                    help="batches of the batched (64) / learned (256) workloads")
    a = ap.parse_args()
    if a.theta is None:
        a.theta = 0.8 if a.workload == "batched" else 0.6
    if a.batches is None:
        a.batches = 256 if a.workload == "learned" else 64
    return a


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d.get("hbm_gbs", HBM_FALLBACK_GBS)), "measured"
    return HBM_FALLBACK_GBS, "fallback"


def profile_traffic(scheme):
    """DRAM bytes per launch of the transaction kernel from a committed ncu
    summary (profiles/ycsb_kernel_<scheme>.txt, line `traffic_per_launch:`)."""
    f = ROOT / "profiles" / f"ycsb_kernel_{scheme}.txt"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        if line.startswith("traffic_per_launch:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


class Clocks:
    """nvidia-smi sampling during the timed region (clocks + throttle reasons)."""

    def __init__(self, dev):
        self.dev, self.proc, self.path = dev, None, None

    def start(self):
        out = Path(os.environ.get("BENCH_CLOCKS_DIR", tempfile.gettempdir()))
        out.mkdir(parents=True, exist_ok=True)
        self.path = out / f"clocks_{os.getpid()}.csv"
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def algorithmic_bytes(txs, row_bytes=88, write_bytes=8):
    """Logical bytes of the committed work (one attempt per tx): the 8 B
    record header + 8 B per request, and per request a 16 B index probe, a
    16 B metadata read + update, then the row read (88 B) or the written
    field (8 B)."""
    cnt = txs["request_cnt"].astype(np.int64)
    mask = np.arange(16)[None, :] < cnt[:, None]
    reads = int((txs["requests"]["read"][mask] != 0).sum())
    ops = int(cnt.sum())
    writes = ops - reads
    return 8 * len(txs) + 8 * ops + reads * (32 + row_bytes) + writes * (32 + write_bytes), reads, writes


def config_of(a):
    return {
        "workload": f"ycsb_plain_{a.rows}rows_{a.txs}tx_16ops_theta{a.theta}_r{a.read_ratio}",
        "cc_scheme": a.scheme, "rows": a.rows, "transactions": a.txs, "ops_per_tx": 16,
        "theta": a.theta, "read_ratio": a.read_ratio, "batch_size": a.batch,
        "warp_density": a.wd, "block_size": a.bs, "layout": "u64 key + 10 u64 fields (88 B, 96 B stride)",
        "write": "fresh uint64 into one uniform field", "index": a.index,
        "l2": "inputs larger than L2 (1.0 GB table + 143 MB transactions > 126 MB L2)",
        "parallelism": f"replicas x{a.gpus}",
        "execution": ("one launch per batch (the reference's batch loop)" if not use_queue(a)
                      else "device queue: one persistent launch drains the batches of "
                           f"{a.batch} in order (GCC_F_QUEUE)"),
    }


# Schemes whose plain runs go through the device queue by default: measured
# on B200 at theta 0.6 (10,485,760 rows, 1,048,576 transactions) the queue
# gives silo 205 -> 237 M and tictoc 206 -> 255 M tx/s; 2PL loses with it
# (tpl_nw 67 -> 46 M: without the batch barrier the hot rows' writers find
# readers in flight at every moment and starve longer) and TO is even.
QUEUE_DEFAULT = ("silo", "tictoc")


def use_queue(a, scheme=None):
    return not a.no_queue and (scheme or a.scheme) in QUEUE_DEFAULT


def cpu_baseline(g, o, txs, a, threads):
    """The CPU executor (oracle port of the CC rules) on the host cores: one
    pass over the whole workload (a fraction of a second to a few seconds on
    16 threads)."""
    n = len(txs)
    sample = txs[:n]
    init = o.fill_table(a.rows, 0, 141919810)
    sch = a.scheme if a.scheme in ("tpl_nw", "silo", "tictoc") else "tpl_nw"
    t, dg, log, secs, aborts = o.cpu_run(sch, init, 0, sample, g.WRITE_FIELD, 1, threads=threads,
                                         commit_log=False)
    nthreads = threads or os.cpu_count()
    return {"value": n / secs if secs > 0 else 0.0, "unit": "tx/s", "cores": nthreads,
            "kind": "port", "scheme": sch,
            "sample": f"first {n} of the {len(txs)} transactions, one pass, {nthreads} threads, "
                      f"{a.rows} rows"}, secs


# Schemes timed against the reference's own GPU build in its own format;
# gacco and mvcc are left out at this shape because the reference's own code
# cannot run them there (oracle/ref_gpu.py: gacco's unbounded hand-off needs
# every transaction of a 65,536-transaction batch resident, MVCC_CPU::Init
# writes past its version array from the second batch on).
REF_GPU_SCHEMES = ("tpl_nw", "tpl_wd", "to", "silo", "tictoc", "gputx", "slow_tpl_nw",
                   "slow_tpl_wd", "slow_to", "slow_silo", "slow_tictoc")


def reference_format_txs(a):
    """The workload's records in the reference's own dataset semantics:
    repeated keys dropped, keys in [1, rows-1] (generation/gen_ycsb.cu)."""
    from oracle import oracle_py as o
    return o.gen_ycsb(a.rows, a.txs, a.theta, a.read_ratio, 141919810, 0, 1)


def reference_gpu_baseline(a, txs):
    """The reference's own test_ycsb (built from its sources into
    oracle/_ref/) on this GPU, per scheme, on `txs` in its own format: 104 B
    rows, sorted-array index, whole-row copies, the same batch size, warp
    density and block size. Its `through` is committed tx over its tot_time
    (metadata resets + precompute + kernels, benchmark_cpu/ycsb.cu:249-291)."""
    from oracle import ref_gpu
    if not ref_gpu.available():
        return {"unavailable": "the reference build is missing (make -C oracle ref REF=<dir>)"}
    out = {"workload": (f"ycsb_ref104_{a.rows}rows_{a.txs}tx_theta{a.theta}_r{a.read_ratio}"
                        f"_batch{a.batch}_wd{a.wd}_bs{a.bs}"),
           "program": "reference test_ycsb (unmodified), NVRTC kernel JIT-compiled for sm_100",
           "tx_per_s": {}, "aborts": {}}
    with tempfile.TemporaryDirectory() as td:
        ds = Path(td) / "ycsb.txs"
        ds.write_bytes(txs.tobytes())
        for s in REF_GPU_SCHEMES:
            try:
                r = ref_gpu.run(ds, a.rows, len(txs), s, a.wd, a.bs, a.batch, timeout=600)
                out["tx_per_s"][s] = r["through"]
                out["aborts"][s] = r.get("abort")
            except Exception as e:  # report, do not fail the engine's line
                out["tx_per_s"][s] = None
                out.setdefault("errors", {})[s] = str(e)[-300:]
    return out


def engine_reference_format(g, a, txs, local, index_kind):
    """The engine on the reference's format and records (the comparison
    side of reference_gpu_baseline): 104 B rows, sorted index, whole-row
    copies, one launch per batch."""
    out = {"tx_per_s": {}, "aborts": {}}
    with g.Engine(a.rows, layout=g.LAYOUT_REF104, index=g.INDEX_SORTED, fill_seed=0,
                  device=local, max_batch=a.batch) as e:
        e.load_txs(txs)
        for s in REF_GPU_SCHEMES:
            k = dict(warp_density=a.wd, block_size=a.bs, batch_size=a.batch,
                     write_mode=g.WRITE_ROWCOPY, write_seed=1)
            e.run(s, **k)
            rs = [e.run(s, **k) for _ in range(3)]
            out["tx_per_s"][s] = statistics.median(r["tx_per_s"] for r in rs)
            out["aborts"][s] = rs[-1]["aborts"]
    return out


CAPS = (128, 256, 512, 1024, 2048)


def learned_vs_plain(g, eng, a, sch, n_batches=16, theta=0.99):
    """The headline comparison, learned scheduling against the plain kernels,
    on the benchmark's table: n_batches batches of 65,536 transactions at Zipf theta 0.99 (read ratio 0.9),
    committed tx/s of
      plain        the plain kernel, one launch per batch, every transaction
                   of the batch in flight the GPU holds;
      plain_best   the plain kernel at its best in-flight cap (max_active
                   swept over CAPS) -- the honest denominator;
      learned      the learned scheduler (predictor trained online, the
                   measured policy, deferral and caps, 2PL lock plans from
                   its key-frequency table) after two training passes;
      untrained    the same scheduler with the network left at its initial
                   weights (train_steps -1): the ablation of the network;
      no_plan      the same scheduler without lock plans (plan_threshold
                   -1): the ablation of the frequency-table lock order."""
    txs = g.gen_ycsb(a.rows, n_batches * a.batch, theta, a.read_ratio, seed=20240521,
                     dedup=g.DEDUP_RESAMPLE, key_base=0)
    eng.load_txs(txs)
    kw = dict(warp_density=a.wd, block_size=a.bs, batch_size=a.batch, write_seed=1)
    out = {"workload": f"ycsb_{a.rows}rows_{n_batches}x{a.batch}tx_16ops_theta{theta}_r{a.read_ratio}",
           "cc_scheme": sch}
    r = eng.run(sch, **kw)
    out["plain"] = {"tx_per_s": r["tx_per_s"], "abort_rate": r["aborts"] / max(1, r["aborts"] + r["committed"])}
    caps = {}
    for c in CAPS:
        eng.run(sch, max_active=c, **kw)
        r = eng.run(sch, max_active=c, **kw)
        caps[c] = r["tx_per_s"]
    best = max(caps, key=caps.get)
    out["plain_caps"] = caps
    out["plain_best"] = {"max_active": best, "tx_per_s": caps[best]}
    for name, steps, plan in (("learned", 0, 0), ("untrained", -1, 0), ("no_plan", 0, -1)):
        with g.Scheduler(eng, mode=g.SCHED_LEARNED, train_steps=steps, seed=7,
                         plan_threshold=plan) as sc:
            sc.run(sch, **kw)
            sc.run(sch, **kw)
            r = sc.run(sch, **kw)
            out[name] = {"tx_per_s": r["committed"] / r["tot_s"],
                         "abort_rate": r["aborts"] / max(1, r["aborts"] + r["committed"]),
                         "p99_us": r["lat_p99_us"]}
    out["learned_over_plain"] = out["learned"]["tx_per_s"] / out["plain"]["tx_per_s"]
    out["learned_over_plain_best"] = out["learned"]["tx_per_s"] / out["plain_best"]["tx_per_s"]
    out["learned_over_untrained"] = out["learned"]["tx_per_s"] / out["untrained"]["tx_per_s"]
    out["learned_over_no_plan"] = out["learned"]["tx_per_s"] / out["no_plan"]["tx_per_s"]
    return out


def run_reference(a):
    """--impl reference: the reference's own implementation of the path,
    timed on this machine. The reference has no CPU execution path (its
    benchmark_cpu/ycsb.cu is the host driver that NVRTC-compiles and
    launches its GPU kernel), so this is its own test_ycsb, compiled from its
    sources into oracle/_ref/ (oracle/Makefile), run unmodified on the
    workload's shape: the same rows, transactions, theta, read ratio, scheme,
    batch_size, warp_density and block_size, in its own record semantics
    (repeated keys dropped, keys 1..rows-1) and row format (104-byte Item
    rows, whole-row copies on write, sorted-array index) -- the only format
    it has. Each step is one test_ycsb run; the value is committed
    transactions over its own tot_time (metadata resets + precompute +
    kernels, benchmark_cpu/ycsb.cu:249-291). The line also carries the
    project's CPU port of the CC rules on all host threads (`cpu_port`).
    It uses nothing of the engine: records come from the oracle's
    generator."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle_py as o
    from oracle import ref_gpu
    threads = a.cpu_threads or os.cpu_count()
    sch = a.scheme
    cfg = config_of(a)
    cfg.update({"layout": "reference Item rows (uint32 id + 10 x char[10] = 104 B)",
                "write": "whole-row copy of the last row read (benchmark/ycsb.cu:57-98)",
                "index": "sorted array (include/index.cuh:65-92)",
                "records": "repeated keys dropped, keys in [1, rows-1] (generation/gen_ycsb.cu)",
                "execution": "the reference's batch loop, one launch per batch"})
    # the project's CPU port of the CC rules, on the engine line's records
    ctx = o.gen_ycsb(a.rows, a.txs, a.theta, a.read_ratio, 141919810, 1, 0)  # dedup resample
    csch = sch if sch in ("tpl_nw", "silo", "tictoc") else "tpl_nw"
    init = o.fill_table(a.rows, 0, 141919810)
    _, _, _, csecs, _ = o.cpu_run(csch, init, 0, ctx, 0, 1, threads=threads, commit_log=False)
    cpu_port = {"value": len(ctx) / csecs, "unit": "tx/s", "cores": threads, "kind": "port",
                "scheme": csch,
                "sample": f"all {len(ctx)} transactions, one pass, {threads} threads, {a.rows} rows"}
    ok, why = ref_gpu.runnable(sch, a.txs, a.wd, a.batch)
    if not ref_gpu.available() or not ok:
        reason = why or "the reference build is missing (make -C oracle ref REF=<dir>)"
        print(json.dumps({"impl": "reference", "unavailable": reason, "cpu_port": cpu_port}),
              flush=True)
        return
    rtx = o.gen_ycsb(a.rows, a.txs, a.theta, a.read_ratio, 141919810, 0, 1)  # dedup drop
    times, walls, aborts = [], [], []
    with tempfile.TemporaryDirectory() as td:
        ds = Path(td) / "ycsb.txs"
        ds.write_bytes(rtx.tobytes())
        try:
            for step in range(a.warmup + a.steps):
                r = ref_gpu.run(ds, a.rows, len(rtx), sch, a.wd, a.bs, a.batch, timeout=600)
                if step >= a.warmup:
                    times.append(r["tot"])
                    walls.append(r["wall_s"])
                    aborts.append(r.get("abort", 0))
        except (RuntimeError, OSError, subprocess.TimeoutExpired) as e:
            # e.g. no GPU on this machine: the reference cannot run at all
            print(json.dumps({"impl": "reference",
                              "unavailable": "the reference's test_ycsb did not run: "
                                             + str(e).splitlines()[0][:200],
                              "cpu_port": cpu_port}), flush=True)
            return
    tot = sum(times)
    v = a.steps * len(rtx) / tot
    line = {"impl": "reference", "metric": "committed tx/s", "value": v, "unit": "tx/s",
            "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": 1000 * tot / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32 keys / byte rows", "data": "synthetic (seeded gen_ycsb semantics)",
            "config": cfg,
            "program": "reference test_ycsb, unmodified (oracle/_ref), its NVRTC kernel "
                       "JIT-compiled for sm_100 by the CUDA driver",
            "aborts_per_step": statistics.mean(aborts),
            "wall_s_per_step": statistics.mean(walls),
            "cpu_baseline": {"value": v, "unit": "tx/s", "cores": 1, "kind": "reference",
                             "sample": f"{len(rtx)} transactions per step; the reference's "
                                       "host driver is one thread and runs its kernel on "
                                       "the GPU (it has no CPU path)"},
            "cpu_port": cpu_port,
            "e2e": {"value": v, "unit": "tx/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def batched_workload(g, a):
    """a.batches batches with log-uniform sizes in [4096, 262144]
    transactions of 4-64 requests (uniform), Zipf theta, read ratio r, on
    the a.rows-row table (seeded)."""
    rng = np.random.default_rng(141919810)
    sizes = np.exp(rng.uniform(np.log(4096), np.log(262144), a.batches)).astype(np.int64)
    boff = np.zeros(a.batches + 1, dtype=np.uint32)
    boff[1:] = np.cumsum(sizes)
    off, reqs = g.gen_ycsb_var(a.rows, int(boff[-1]), a.theta, a.read_ratio, min_ops=4,
                               max_ops=64, seed=141919810)
    return boff, off, reqs


def run_batched(a):
    """Uneven batched workload: the device-queue executor (one persistent
    kernel, CUDA graph, autotuned) against the same batches launched one by
    one with plain kernels, and one by one with the per-batch tuner."""
    from gpu_cc_tb_b200 import replicas
    rank, ws, local, dist = replicas.init_from_env("nccl")
    import torch
    import gpu_cc_tb_b200 as g
    boff, off, reqs = batched_workload(g, a)
    n_tx, n_ops = len(off) - 1, int(off[-1])
    reads = int(reqs["read"].sum())
    alg = 8 * n_tx + 8 * n_ops + reads * (32 + 88) + (n_ops - reads) * (32 + 8)
    pinned = torch.empty(reqs.nbytes, dtype=torch.uint8, pin_memory=True)
    host_reqs = pinned.numpy().view(g.REQ_DTYPE)
    host_reqs[:] = reqs
    eng = g.Engine(a.rows, layout=g.LAYOUT_U64X11, index=g.INDEX_HASH, fill_seed=141919810,
                   device=local, max_batch=int(np.diff(boff).max()))
    eng.load_var_txs(off, host_reqs)
    sch = a.scheme
    tuned = dict(warp_density=a.wd, block_size=a.bs, flags=g.F_AUTOTUNE | g.F_GRAPH, write_seed=1)
    plain = dict(warp_density=a.wd, block_size=a.bs, flags=0, write_seed=1)
    warm_tuned = max(a.warmup, 9)  # the tuner measures its 8 arms, then settles
    for _ in range(warm_tuned):
        eng.run_batches(sch, boff, g.BATCHES_QUEUE, **tuned)
    clocks = Clocks(local)
    replicas.barrier(dist)
    clocks.start()
    dev_s, committed, aborts, kern_ms = 0.0, 0, 0, 0.0
    lat50, lat99 = [], []
    for _ in range(a.steps):
        r = eng.run_batches(sch, boff, g.BATCHES_QUEUE, **tuned)
        dev_s += r["tot_s"]
        committed += r["committed"]
        aborts += r["aborts"]
        kern_ms += r["proc_s"] * 1000
        lat50.append(r["lat_p50_us"])
        lat99.append(r["lat_p99_us"])
    replicas.barrier(dist)
    clk = clocks.stop()
    wd_q, bs_q, _ = eng.batch_stats()
    act_q = eng.batch_active()
    # the same batches one by one, plain kernels at the given knobs
    for _ in range(min(a.warmup, 1)):
        eng.run_batches(sch, boff, g.BATCHES_SEQUENTIAL, **plain)
    base_s, base_c, base_launch = 0.0, 0, 0
    for _ in range(a.steps):
        r = eng.run_batches(sch, boff, g.BATCHES_SEQUENTIAL, **plain)
        base_s += r["tot_s"]
        base_c += r["committed"]
        base_launch += r["kernel_launches"]
    # one by one with the per-batch-class tuner and graph replay
    for _ in range(warm_tuned):
        eng.run_batches(sch, boff, g.BATCHES_SEQUENTIAL, **tuned)
    seq_s, seq_c = 0.0, 0
    for _ in range(a.steps):
        r = eng.run_batches(sch, boff, g.BATCHES_SEQUENTIAL, **tuned)
        seq_s += r["tot_s"]
        seq_c += r["committed"]
    # end to end through the public API: H2D of the requests from pinned
    # memory, the queue run, D2H of every transaction's read digest
    e2e_s = 0.0
    dig = torch.empty(n_tx * 8, dtype=torch.uint8, pin_memory=True).numpy().view(np.uint64)
    for _ in range(a.steps):
        replicas.barrier(dist)
        s0 = time.perf_counter()
        eng.load_var_txs(off, host_reqs)
        eng.run_batches(sch, boff, g.BATCHES_QUEUE, **tuned)
        g.library().gcc_get_digests(eng._h, g.C.c_void_p(dig.ctypes.data), n_tx)
        e2e_s += time.perf_counter() - s0
    job = replicas.combine(dist, dev_s, committed, e2e_s, a.steps * n_tx)
    if rank == 0:
        hbm, kind = peaks()
        launch_ms = kern_ms / a.steps
        achieved = alg / (launch_ms / 1000) / 1e9
        line = {
            "metric": "committed tx/s", "value": job["value"], "unit": "tx/s", "n_gpus": ws,
            "steps": a.steps, "warmup": warm_tuned,
            "ms_per_step": 1000 * job["device_s_max"] / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic (seeded variable-length gen_ycsb)",
            "config": {"workload": f"ycsb_batched_{a.batches}_uneven_batches_{n_tx}tx_4to64ops_"
                                   f"theta{a.theta}_r{a.read_ratio}",
                       "cc_scheme": sch, "rows": a.rows, "transactions": n_tx, "requests": n_ops,
                       "batch_sizes": "log-uniform in [4096, 262144]", "ops_per_tx": "uniform 4-64",
                       "theta": a.theta, "read_ratio": a.read_ratio,
                       "executor": "one persistent kernel, device queue, CUDA graph, autotuned",
                       "tuned_config": {"warp_density": int(wd_q[0]), "block_size": int(bs_q[0]),
                                        "in_flight": int(act_q[0])},
                       "l2": "inputs larger than L2 (1.0 GB table + requests)",
                       "parallelism": f"replicas x{ws}"},
            "one_by_one_plain": {"value": base_c / base_s, "unit": "tx/s",
                                 "kernel_launches_per_step": base_launch // a.steps,
                                 "config": {"warp_density": a.wd, "block_size": a.bs}},
            "one_by_one_autotuned_graph": {"value": seq_c / seq_s, "unit": "tx/s"},
            "speedup_vs_one_by_one_plain": (committed / dev_s) / (base_c / base_s),
            "aborts_per_step": aborts / a.steps,
            "abort_rate": aborts / max(1, aborts + committed),
            "latency_us": {"p50": statistics.median(lat50), "p99": statistics.median(lat99)},
            "e2e": {"value": job["e2e_value"], "unit": "tx/s",
                    "h2d_bytes_per_step": int(reqs.nbytes + off.nbytes),
                    "d2h_bytes_per_step": int(n_tx * 8)},
            "gpu_launches": 3 * a.steps,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "traffic": None, "kernel": "ycsb_kernel (queue)",
                         "peak_kind": kind, "alg_bytes_per_launch": alg, "launch_ms": launch_ms},
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    eng.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def learned_workload(g, a):
    """a.batches batches of 65,536 x 16-request transactions; theta drifts
    linearly 0.5 -> 0.99 and the read ratio 0.9 -> 0.5 across batches."""
    parts = []
    nb = a.batches
    for b in range(nb):
        f = b / max(1, nb - 1)
        parts.append(g.gen_ycsb(a.rows, a.batch, 0.5 + 0.49 * f, 0.9 - 0.4 * f, seed=141919810 + b,
                                dedup=g.DEDUP_RESAMPLE, key_base=0))
    return np.concatenate(parts)


def run_learned(a):
    """Learned contention scheduling against plain ordering on identical
    batches, both through gcc_sched_run (the plain arm runs no predictor)."""
    from gpu_cc_tb_b200 import replicas
    rank, ws, local, dist = replicas.init_from_env("nccl")
    import torch
    import gpu_cc_tb_b200 as g
    sch = a.scheme if a.scheme in g.SCHED_SCHEMES else "tpl_nw"
    txs = learned_workload(g, a)
    n = len(txs)
    pinned = torch.empty(txs.nbytes, dtype=torch.uint8, pin_memory=True)
    host_txs = pinned.numpy().view(g.TX_DTYPE)
    host_txs[:] = txs
    eng = g.Engine(a.rows, layout=g.LAYOUT_U64X11, index=g.INDEX_HASH, fill_seed=141919810,
                   device=local, max_batch=a.batch)
    eng.load_txs(host_txs)
    kw = dict(warp_density=a.wd, block_size=a.bs, batch_size=a.batch, write_seed=1)
    learned = g.Scheduler(eng, mode=g.SCHED_LEARNED, seed=7)
    plain = g.Scheduler(eng, mode=g.SCHED_PLAIN)
    for _ in range(a.warmup):
        learned.run(sch, **kw)          # trains the network, settles the policy
    plain.run(sch, **kw)
    clocks = Clocks(local)
    replicas.barrier(dist)
    clocks.start()
    dev_s, committed, aborts, launches, lat99 = 0.0, 0, 0, 0, []
    res = []
    for _ in range(a.steps):
        r = learned.run(sch, **kw)
        dev_s += r["tot_s"]
        committed += r["committed"]
        aborts += r["aborts"]
        launches += r["kernel_launches"]
        lat99.append(r["lat_p99_us"])
        res.append(r)
    replicas.barrier(dist)
    clk = clocks.stop()
    recs = learned.batches()
    p_s, p_c, p_a, p_lat = 0.0, 0, 0, []
    for _ in range(a.steps):
        r = plain.run(sch, **kw)
        p_s += r["tot_s"]
        p_c += r["committed"]
        p_a += r["aborts"]
        p_lat.append(r["lat_p99_us"])
    # the high-contention end: the last quarter of the batches (theta >= 0.87)
    q0 = 3 * len(recs) // 4
    hi_l = sum(b["committed"] for b in recs[q0:]) / (sum(b["ms"] for b in recs[q0:]) / 1e3)
    precs = plain.batches()
    hi_p = sum(b["committed"] for b in precs[q0:]) / (sum(b["ms"] for b in precs[q0:]) / 1e3)
    e2e_s = 0.0
    dig = torch.empty(n * 8, dtype=torch.uint8, pin_memory=True).numpy().view(np.uint64)
    for _ in range(a.steps):
        replicas.barrier(dist)
        s0 = time.perf_counter()
        eng.load_txs(host_txs)
        learned.run(sch, **kw)
        g.library().gcc_get_digests(eng._h, g.C.c_void_p(dig.ctypes.data), n)
        e2e_s += time.perf_counter() - s0
    job = replicas.combine(dist, dev_s, committed, e2e_s, a.steps * n)
    if rank == 0:
        last = res[-1]
        hbm, kind = peaks()
        alg, _, _ = algorithmic_bytes(txs)
        kern_s = sum(r["proc_s"] for r in res) / a.steps
        achieved = alg / kern_s / 1e9
        line = {
            "metric": "committed tx/s (learned vs plain CC, same GPU, 0 violations)",
            "value": job["value"], "unit": "tx/s", "n_gpus": ws, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": 1000 * job["device_s_max"] / a.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic (seeded gen_ycsb per batch)",
            "config": {"workload": f"ycsb_learned_{a.batches}x{a.batch}tx_16ops_theta0.5to0.99_"
                                   f"r0.9to0.5", "cc_scheme": sch, "rows": a.rows,
                       "transactions": n, "batch_size": a.batch, "warp_density": a.wd,
                       "block_size": a.bs,
                       "predictor": "MLP 66-128-128-1, BF16 weights, FP32 accumulation, "
                                    "trained online on probe abort labels",
                       "l2": "inputs larger than L2 (1.0 GB table + 2.3 GB transactions)",
                       "parallelism": f"replicas x{ws}"},
            "plain_ordering": {"value": p_c / p_s, "unit": "tx/s",
                               "abort_rate": p_a / max(1, p_a + p_c),
                               "p99_us": statistics.median(p_lat)},
            "speedup_vs_plain": (committed / dev_s) / (p_c / p_s),
            "high_contention_quarter": {"theta": ">= 0.87", "learned_tx_per_s": hi_l,
                                        "plain_tx_per_s": hi_p, "speedup": hi_l / hi_p},
            "abort_rate": aborts / max(1, aborts + committed),
            "probe_abort_rate": last["probe_abort_rate"],
            "sched_abort_rate": last["sched_abort_rate"],
            "predictor": {"predict_ms": last["predict_ms"], "train_ms": last["train_ms"],
                          "last_probe_loss": last["last_loss"]},
            "latency_us": {"p99": statistics.median(lat99)},
            "e2e": {"value": job["e2e_value"], "unit": "tx/s", "h2d_bytes_per_step": int(txs.nbytes),
                    "d2h_bytes_per_step": int(n * 8)},
            "gpu_launches": int(launches // a.steps),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "traffic": None,
                         "kernel": "ycsb_kernel (all launches of a pass)", "peak_kind": kind,
                         "alg_bytes_per_pass": alg, "kernel_s_per_pass": kern_s},
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    learned.close()
    plain.close()
    eng.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def serving_cpu_baseline(g, d, off, reqs, sch, a, n=200_000):
    """The CPU executors (oracle port of the CC rules, all host threads) on
    the first n order-entry transactions, closed loop (all arrived)."""
    try:
        from oracle import oracle_py as o
        tx_off = np.ascontiguousarray(off[:n + 1])
        rq = reqs[:int(off[n])]
        lay_rows = int(rq["key"].max()) + 1
        init = o.fill_table(lay_rows, g.LAYOUT_U64X11, 141919810)
        kind = sch if sch in ("tpl_nw", "silo", "tictoc") else "tpl_nw"
        threads = a.cpu_threads or os.cpu_count()
        _, _, _, secs, aborts = o.cpu_run_var(kind, init, g.LAYOUT_U64X11, tx_off, rq,
                                              g.WRITE_FIELD, 1, ext_ops=True, threads=threads,
                                              commit_log=False)
        return {"value": n / secs if secs > 0 else 0.0, "unit": "tx/s", "cores": threads,
                "kind": "port", "scheme": kind, "aborts": int(aborts),
                "sample": f"first {n} order-entry transactions, closed loop, {threads} threads"}
    except Exception as ex:  # the GPU line stays valid without it
        return {"error": str(ex)[:200]}


def run_serving(a):
    """Order-entry serving: peak (saturated) commits/s and a Poisson load
    sweep with p50/p99 latency, learned scheduler on vs off."""
    from gpu_cc_tb_b200 import replicas
    rank, ws, local, dist = replicas.init_from_env("nccl")
    import torch  # noqa: F401  (CUDA context for the replicas' barrier)
    import gpu_cc_tb_b200 as g
    sch = a.scheme if a.scheme in g.SCHED_SCHEMES else "tpl_nw"
    d = g.order_entry_desc()
    n_all = 1_500_000
    off, reqs, kind, lay = g.gen_order_entry(d, n_all, seed=141919810)
    eng = g.Engine(lay["rows"], layout=g.LAYOUT_U64X11, index=g.INDEX_DIRECT, fill_seed=0,
                   device=local, max_batch=65536)
    eng.oe_fill(d, seed=141919810)
    kw = dict(warp_density=a.wd, block_size=a.bs, flags=g.F_EXT_OPS | g.F_NO_RESET, write_seed=1)

    def load(n):
        eng.load_var_txs(off[:n + 1], reqs[:int(off[n])])

    on = g.Scheduler(eng, mode=g.SCHED_LEARNED, seed=7)
    off_s = g.Scheduler(eng, mode=g.SCHED_PLAIN)
    n_peak = 600_000
    load(n_peak)
    for _ in range(max(1, a.warmup)):
        on.serve(sch, rate_tps=1e10, seed=1, max_batch=65536, **kw)   # trains, settles
        off_s.serve(sch, rate_tps=1e10, seed=1, max_batch=65536, **kw)
    clocks = Clocks(local)
    replicas.barrier(dist)
    clocks.start()
    peak = {"on": [], "off": []}
    dev = {"on": [], "off": []}
    launches = 0
    for _ in range(a.steps):
        r = on.serve(sch, rate_tps=1e10, seed=2, max_batch=65536, **kw)
        launches += r["kernel_launches"]
        peak["on"].append(r["tx_per_s"])
        dev["on"].append(r["device_tx_per_s"])
        r = off_s.serve(sch, rate_tps=1e10, seed=2, max_batch=65536, **kw)
        peak["off"].append(r["tx_per_s"])
        dev["off"].append(r["device_tx_per_s"])
    replicas.barrier(dist)
    clk = clocks.stop()
    p_on, p_off = statistics.median(peak["on"]), statistics.median(peak["off"])
    # end to end: upload of the request stream + saturated serving
    e2e_s = 0.0
    for _ in range(a.steps):
        s0 = time.perf_counter()
        load(n_peak)
        on.serve(sch, rate_tps=1e10, seed=3, max_batch=65536, **kw)
        e2e_s += time.perf_counter() - s0
    # Poisson load sweep relative to the plain peak
    sweep = []
    for frac in (0.1, 0.25, 0.5, 0.75, 0.9, 1.0, 1.2):
        rate = frac * p_off
        n = int(min(n_all, max(20_000, rate * 1.5)))
        load(n)
        pt = {"load": frac, "rate_tps": rate, "transactions": n}
        for name, sc in (("on", on), ("off", off_s)):
            r = sc.serve(sch, rate_tps=rate, seed=11, max_batch=65536, **kw)
            pt[name] = {"tx_per_s": r["tx_per_s"], "p50_us": r["lat_p50_us"],
                        "p99_us": r["lat_p99_us"], "mean_batch": r["mean_batch"],
                        "abort_rate": r["sched_abort_rate"]}
        sweep.append(pt)
    job = replicas.combine(dist, n_peak * a.steps / p_on, n_peak * a.steps, e2e_s, a.steps * n_peak)
    if rank == 0:
        cpu = serving_cpu_baseline(g, d, off, reqs, sch, a)
        line = {
            "metric": "committed tx/s (learned vs plain CC, same GPU, 0 violations); p99",
            "value": job["value"], "unit": "tx/s", "n_gpus": ws, "steps": a.steps,
            "warmup": max(1, a.warmup), "ms_per_step": 1000 * n_peak / p_on,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic (seeded order-entry generator, Poisson arrivals)",
            "config": {"workload": "order_entry_serving_W64_D10_C3000_I100000_50no_50pay",
                       "cc_scheme": sch, "rows": lay["rows"], "warp_density": a.wd,
                       "block_size": a.bs, "peak_transactions": n_peak,
                       "admission": "all arrived, at most 65,536 per batch",
                       "state": "table and CC metadata resident (no per-batch reset)",
                       "parallelism": f"replicas x{ws}"},
            "peak": {"learned_tx_per_s": p_on, "plain_tx_per_s": p_off,
                     "speedup": p_on / p_off,
                     "learned_device_tx_per_s": statistics.median(dev["on"]),
                     "plain_device_tx_per_s": statistics.median(dev["off"])},
            "sweep": sweep,
            "e2e": {"value": job["e2e_value"], "unit": "tx/s",
                    "h2d_bytes_per_step": int(reqs[:int(off[n_peak])].nbytes + 4 * (n_peak + 1)),
                    "d2h_bytes_per_step": 0},
            "gpu_launches": int(launches // a.steps),
            "cpu_baseline": cpu,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    on.close()
    off_s.close()
    eng.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def run_sweep(a):
    """The plain-YCSB scheme sweep on one B200: every scheme x theta {0.1, 0.6, 0.8, 0.99} x read ratio
    {1.0, 0.9, 0.5} at warp_density 5 / block_size 32, and the warp_density
    0-5 x block_size {1, 8, 16, 32} grid at theta 0.6 and 0.99 (tpl_nw and
    silo), on 10,485,760 rows with --txs transactions of 16 requests in
    batches of --batch; per point committed tx/s (the reference's tot_time
    definition), aborted attempts and algorithmic GB/s of the transaction
    kernel. Then the reference's own dataset points in its own format
    (104 B rows, sorted index, whole-row copies, batch 1,048,576): ro (theta
    0, reads only), mc (theta 0.6, r 0.9), hc (theta 0.8, r 0.5) and t9
    (theta 0.9, r 0.9, the highest contention the reference publishes), for
    the engine and for the reference's GPU build (not at theta 0.99: its
    retries are immediate and unbounded, and its published runs stop at
    0.9). One JSON line per point, then the summary line. The scheme grid
    uses --sweep-txs transactions per point, the reference points --txs."""
    from gpu_cc_tb_b200 import replicas
    rank, ws, local, dist = replicas.init_from_env("nccl")
    import gpu_cc_tb_b200 as g
    hbm, kind = peaks()
    clocks = Clocks(local)
    clocks.start()
    points = []

    def point(eng, txs, alg, s, theta, r, wd, bs, extra=None):
        k = dict(warp_density=wd, block_size=bs, batch_size=a.batch, write_seed=1)
        if s in QUEUE_DEFAULT and not a.no_queue:
            k["flags"] = g.F_QUEUE
        try:
            eng.run(s, **k)
            res = eng.run(s, **k)
            km, _ = eng.last_kernel_ms()
            pt = {"scheme": s, "theta": theta, "read_ratio": r, "wd": wd, "bs": bs,
                  "tx_per_s": res["tx_per_s"], "aborts": res["aborts"],
                  "alg_gbs": alg / (km / 1e3) / 1e9 if km > 0 else None,
                  "p99_us": res["lat_p99_us"], "queue": bool(k.get("flags", 0))}
        except g.GccError as e:
            pt = {"scheme": s, "theta": theta, "read_ratio": r, "wd": wd, "bs": bs,
                  "error": str(e)}
        if extra:
            pt.update(extra)
        points.append(pt)
        if rank == 0:
            print(json.dumps(pt), flush=True)

    with g.Engine(a.rows, layout=g.LAYOUT_U64X11, index=g.INDEX_HASH, fill_seed=141919810,
                  device=local, max_batch=a.batch) as eng:
        for theta in ((0.1, 0.6, 0.8, 0.99) if a.sweep_grid else ()):
            for r in (1.0, 0.9, 0.5):
                txs = g.gen_ycsb(a.rows, a.sweep_txs, theta, r, seed=141919810,
                                 dedup=g.DEDUP_RESAMPLE, key_base=0)
                alg, _, _ = algorithmic_bytes(txs)
                eng.load_txs(txs)
                for s in g.SCHEMES:
                    point(eng, txs, alg, s, theta, r, 5, 32)
                if r == 0.9 and theta in (0.6, 0.99):
                    for s in ("tpl_nw", "silo"):
                        for wd in range(6):
                            for bs in (1, 8, 16, 32):
                                if (wd, bs) != (5, 32):
                                    point(eng, txs, alg, s, theta, r, wd, bs, {"grid": True})
    # the reference's dataset points, engine and reference build side by side
    ref_points = {}
    from oracle import ref_gpu
    for name, theta, r in (("ro", 0.0, 1.0), ("mc", 0.6, 0.9), ("hc", 0.8, 0.5), ("t9", 0.9, 0.9)):
        if name not in a.ref_points.split(","):
            continue
        etx = g.gen_ycsb(a.rows, a.txs, theta, r, seed=141919810, dedup=g.DEDUP_DROP, key_base=1)
        rp = {"engine": {}, "reference": {}}
        with g.Engine(a.rows, layout=g.LAYOUT_REF104, index=g.INDEX_SORTED, fill_seed=0,
                      device=local, max_batch=a.txs) as e:
            e.load_txs(etx)
            for s in g.SCHEMES:
                k = dict(warp_density=5, block_size=32, batch_size=a.txs,
                         write_mode=g.WRITE_ROWCOPY, write_seed=1)
                try:
                    e.run(s, **k)
                    rp["engine"][s] = e.run(s, **k)["tx_per_s"]
                except g.GccError as ex:
                    rp["engine"][s] = str(ex)
        if ref_gpu.available():
            from oracle import oracle_py as o
            rtx = o.gen_ycsb(a.rows, a.txs, theta, r, 141919810, 0, 1)
            with tempfile.TemporaryDirectory() as td:
                ds = Path(td) / f"{name}.txs"
                ds.write_bytes(rtx.tobytes())
                for s in g.SCHEMES:
                    ok, why = ref_gpu.runnable(s, a.txs, 5, a.txs)
                    if not ok:
                        rp["reference"][s] = f"not run: {why}"
                        continue
                    try:
                        rp["reference"][s] = ref_gpu.run(ds, a.rows, a.txs, s, 5, 32, a.txs,
                                                         timeout=600)["through"]
                    except Exception as ex:
                        rp["reference"][s] = f"error: {str(ex)[-200:]}"
        ref_points[name] = rp
        if rank == 0:
            print(json.dumps({"ref_point": name, **rp}), flush=True)
    clk = clocks.stop()
    if rank == 0:
        best = {}
        for pt in points:
            if "tx_per_s" in pt and not pt.get("grid"):
                best[f"{pt['scheme']}_t{pt['theta']}_r{pt['read_ratio']}"] = pt["tx_per_s"]
        print(json.dumps({"metric": "committed tx/s", "workload": "plain YCSB scheme sweep",
                          "unit": "tx/s", "rows": a.rows, "transactions": a.sweep_txs,
                          "reference_point_transactions": a.txs,
                          "batch_size": a.batch, "points": len(points), "by_point": best,
                          "reference_points": ref_points, "hbm_peak_gbs": hbm,
                          "peak_kind": kind, "clocks": clk}), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
        return
    if a.workload == "batched":
        run_batched(a)
        return
    if a.workload == "learned":
        run_learned(a)
        return
    if a.workload == "serving":
        run_serving(a)
        return
    if a.workload == "sweep":
        run_sweep(a)
        return
    from gpu_cc_tb_b200 import replicas
    rank, ws, local, dist = replicas.init_from_env("nccl")
    import torch
    import gpu_cc_tb_b200 as g
    index = {"hash": g.INDEX_HASH, "sorted": g.INDEX_SORTED, "direct": g.INDEX_DIRECT}[a.index]

    txs = g.gen_ycsb(a.rows, a.txs, a.theta, a.read_ratio, seed=141919810,
                     dedup=g.DEDUP_RESAMPLE, key_base=0)
    alg_bytes, reads, writes = algorithmic_bytes(txs)
    # pinned host copy of the transactions for the end-to-end leg
    pinned = torch.empty(txs.nbytes, dtype=torch.uint8, pin_memory=True)
    host_txs = pinned.numpy().view(g.TX_DTYPE)
    host_txs[:] = txs
    digests_host = torch.empty(a.txs * 8, dtype=torch.uint8, pin_memory=True).numpy().view(np.uint64)

    eng = g.Engine(a.rows, layout=g.LAYOUT_U64X11, index=index, fill_seed=141919810,
                   device=local, max_batch=a.batch)
    eng.load_txs(host_txs)
    flags = (g.F_NO_RESET if a.no_reset else 0) | (g.F_QUEUE if use_queue(a) else 0)
    kw = dict(warp_density=a.wd, block_size=a.bs, batch_size=a.batch, flags=flags, write_seed=1)
    for _ in range(a.warmup):
        eng.run(a.scheme, **kw)

    clocks = Clocks(local)
    replicas.barrier(dist)
    clocks.start()
    dev_s, kern_ms, launches, committed, aborts = 0.0, 0.0, 0, 0, 0
    lat50, lat99 = [], []
    t0 = time.perf_counter()
    for _ in range(a.steps):
        r = eng.run(a.scheme, **kw)
        dev_s += r["tot_s"]
        km, _ = eng.last_kernel_ms()
        kern_ms += km
        launches += r["kernel_launches"]
        committed += r["committed"]
        aborts += r["aborts"]
        lat50.append(r["lat_p50_us"])
        lat99.append(r["lat_p99_us"])
        n_tx_launches = r["batches"]
    wall = time.perf_counter() - t0
    replicas.barrier(dist)

    # end to end through the public API: H2D of the step's transactions from
    # pinned memory, the run, D2H of every transaction's read digest; the
    # engine overlaps each batch's copies with the other batches' execution
    # (gcc_run_host). The clock record covers both timed regions.
    for _ in range(a.warmup):
        eng.run_host(a.scheme, host_txs, digests_host, **kw)
    e2e_s = 0.0
    for _ in range(a.steps):
        replicas.barrier(dist)
        s0 = time.perf_counter()
        eng.run_host(a.scheme, host_txs, digests_host, **kw)
        e2e_s += time.perf_counter() - s0
    clk = clocks.stop()

    job = replicas.combine(dist, dev_s, committed, e2e_s, a.steps * a.txs)
    dev_s_max, value, e2e_val = job["device_s_max"], job["value"], job["e2e_value"]

    if rank == 0:
        hbm, kind = peaks()
        launch_ms = kern_ms / (a.steps * n_tx_launches)
        per_launch_bytes = alg_bytes / n_tx_launches
        achieved = per_launch_bytes / (launch_ms / 1000) / 1e9
        traffic = profile_traffic(a.scheme)
        line = {
            "metric": "committed tx/s", "value": value, "unit": "tx/s", "n_gpus": ws,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1000 * dev_s_max / a.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic (seeded gen_ycsb, counter-based RNG)",
            "config": config_of(a),
            "aborts_per_step": aborts / a.steps,
            "abort_rate": aborts / max(1, aborts + committed),
            "latency_us": {"p50": statistics.median(lat50), "p99": statistics.median(lat99)},
            "wall_s": wall,
            "e2e": {"value": e2e_val, "unit": "tx/s", "h2d_bytes_per_step": int(txs.nbytes),
                    "d2h_bytes_per_step": int(a.txs * 8)},
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "traffic": traffic,
                         "kernel": "ycsb_kernel", "peak_kind": kind,
                         "alg_bytes_per_launch": per_launch_bytes,
                         "launch_ms": launch_ms},
            "clocks": clk,
        }
        if not a.no_cpu_baseline and ws == 1:
            from oracle import oracle_py as o
            line["cpu_baseline"], _ = cpu_baseline(g, o, txs, a, a.cpu_threads)
        if ws == 1:
            # the reference's CPU-runnable shape (1,048,576 rows, 65,536
            # transactions, theta 0.1, one batch): the same kernel at low
            # contention, for the roofline
            c0 = g.gen_ycsb(1_048_576, 65_536, 0.1, a.read_ratio, seed=141919810,
                            dedup=g.DEDUP_RESAMPLE, key_base=0)
            b0, _, _ = algorithmic_bytes(c0)
            with g.Engine(1_048_576, layout=g.LAYOUT_U64X11, index=index, fill_seed=141919810,
                          device=local, max_batch=65_536) as e0:
                e0.load_txs(c0)
                k0 = dict(kw, batch_size=65_536)
                for _ in range(3):
                    e0.run(a.scheme, **k0)
                rs = [e0.run(a.scheme, **k0) for _ in range(5)]
                kms = e0.last_kernel_ms()[0]
            ach = b0 / (kms / 1000) / 1e9
            line["config0"] = {"workload": "ycsb_plain_1048576rows_65536tx_16ops_theta0.1_r0.9",
                               "tx_per_s": statistics.median(r["tx_per_s"] for r in rs),
                               "kernel_ms": kms, "achieved_gbs": ach, "frac_of_hbm": ach / hbm,
                               "note": "one launch of 65,536 transactions at low contention"}
        if use_queue(a):
            # the same workload with one launch per batch, for comparison
            ks = dict(kw, flags=kw["flags"] & ~g.F_QUEUE)
            eng.run(a.scheme, **ks)
            rs = [eng.run(a.scheme, **ks) for _ in range(3)]
            line["per_batch_launches"] = {
                "tx_per_s": statistics.median(r["tx_per_s"] for r in rs),
                "launches": rs[0]["batches"],
                "note": "same workload, one kernel launch per 65,536-transaction batch"}
        if a.sweep:
            sw = {}
            for s in a.sweep.split(","):
                fl = kw["flags"] & ~g.F_QUEUE
                if use_queue(a, s):
                    fl |= g.F_QUEUE
                ks = dict(kw, flags=fl)
                eng.run(s, **ks)          # first run sizes the scheme's buffers
                r = eng.run(s, **ks)
                sw[s] = {"tx_per_s": r["tx_per_s"], "aborts": r["aborts"],
                         "p99_us": r["lat_p99_us"], "queue": bool(fl & g.F_QUEUE)}
            line["sweep"] = sw
        if ws == 1 and not a.no_learned and a.scheme in g.SCHED_SCHEMES:
            line["learned_vs_plain"] = learned_vs_plain(g, eng, a, a.scheme)
        if ws == 1 and not a.no_reference_gpu:
            ref = reference_gpu_baseline(a, reference_format_txs(a))
            line["reference_gpu"] = ref
            if "tx_per_s" in ref:
                # the same records from the engine's own generator
                etx = g.gen_ycsb(a.rows, a.txs, a.theta, a.read_ratio, seed=141919810,
                                 dedup=g.DEDUP_DROP, key_base=1)
                eng_ref = engine_reference_format(g, a, etx, local, index)
                line["engine_reference_format"] = eng_ref
                line["vs_reference_gpu"] = {
                    s: (eng_ref["tx_per_s"][s] / ref["tx_per_s"][s]
                        if ref["tx_per_s"].get(s) else None) for s in REF_GPU_SCHEMES}
        print(json.dumps(line), flush=True)
    eng.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
