"""Runs the reference's own test_ycsb on the GPU (built from the reference's
sources into oracle/_ref/ by `make -C oracle ref REF=<reference dir>`).

TEST INFRASTRUCTURE and the reference arm of bench.py: the engine never
calls it. It runs
  * _ref/test_ycsb       -- the reference's host driver, unmodified, in
                            _ref/run/ (it NVRTC-compiles ./benchmark/ycsb.cu,
                            benchmark_cpu/ycsb.cu:86-88,203-226), or
  * _ref/test_ycsb_dump  -- the same driver with zero-initialised rows and
                            `Item item`, writing the final table to a file
                            (see oracle/Makefile), in _ref/run_dump/,
with the reference's argv (readme.md:62-70):
    test_ycsb <dataset> <rows> <txcnt> <cc_scheme> <warp_density>
              <block_size> <batch_size> <debug>
and parses the report block of ExecInfo::Analyse (include/runtime.cuh:
198-213). NVRTC writes the compiled kernel to out/bench_ycsb.ptx
(include/env.cuh:156-159); that file is deleted unread after every run.

Runs that cannot finish are never started (the caller checks with
`runnable`): the reference's waits are unbounded, so
  * gacco needs every transaction of a batch resident at once (a
    transaction spins until every lower one in its object's queue has
    passed, include/gacco.cuh:156-175): batch x 2^warp_density threads must
    fit in one wave of 1,024-thread CTAs, one per SM;
  * mvcc / slow_mvcc with more than one batch memset past the end of the
    version-node array (MVCC_CPU::Init adds sizeof(version_node) * offset to
    a version_node pointer, include/mvcc.cuh:361-374), so they run only with
    batch_size >= txcnt.
"""
from __future__ import annotations

import os
import re
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
REF = HERE / "_ref"
ONE_WAVE_THREADS = 148 * 1024  # one 1,024-thread CTA per SM on a B200

_NUM = re.compile(r"^(through|abort|ts_d|wait_d|abort_d|mng_d|tot_d|idx_d|pre|proc|tot) "
                  r"(-?[0-9.eE+-]+|inf|nan)")


def available(dump: bool = False) -> bool:
    exe = REF / ("test_ycsb_dump" if dump else "test_ycsb")
    run = REF / ("run_dump" if dump else "run")
    return exe.exists() and (run / "benchmark" / "ycsb.cu").exists() and (run / "include").is_dir()


def runnable(scheme: str, n_tx: int, warp_density: int, batch_size: int) -> tuple[bool, str]:
    """Whether a reference run of this shape is known to finish (see the
    module docstring); (False, reason) otherwise."""
    batch = min(batch_size, n_tx)
    if scheme == "gacco" and batch * (1 << warp_density) > ONE_WAVE_THREADS:
        return False, ("gacco's hand-off waits on lower transactions of the batch without a "
                       "bound; a batch larger than one wave of CTAs may wait on one that is "
                       "not resident")
    if scheme in ("mvcc", "slow_mvcc", "slowmvcc") and batch < n_tx:
        return False, ("MVCC_CPU::Init memsets past the version-node array from the second "
                       "batch on (include/mvcc.cuh:361-374)")
    return True, ""


def _clear_ptx(run_dir: Path):
    out = run_dir / "out"
    if out.is_dir():
        for f in out.iterdir():
            if f.is_file():
                f.unlink()  # compiler-written code: deleted unread


def run(dataset: Path, rows: int, n_tx: int, scheme: str, warp_density: int = 5,
        block_size: int = 32, batch_size: int = 65536, dump_table: Path | None = None,
        timeout: float = 900.0) -> dict:
    """One test_ycsb run; returns the report's numbers (through = committed
    tx/s by the reference's own tot_time, abort = aborted attempts, pre /
    proc / tot = seconds) plus wall seconds."""
    ok, why = runnable(scheme, n_tx, warp_density, batch_size)
    if not ok:
        raise ValueError(f"reference run not started: {why}")
    dump = dump_table is not None
    if not available(dump):
        raise FileNotFoundError(f"reference build missing under {REF} (make -C oracle ref)")
    exe = REF / ("test_ycsb_dump" if dump else "test_ycsb")
    cwd = REF / ("run_dump" if dump else "run")
    (cwd / "out").mkdir(exist_ok=True)
    env = dict(os.environ)
    if dump:
        env["GCC_REF_TABLE_OUT"] = str(dump_table)
    cmd = [str(exe), str(dataset), str(rows), str(n_tx), scheme, str(warp_density),
           str(block_size), str(batch_size), "0"]
    import time
    t0 = time.perf_counter()
    try:
        r = subprocess.run(cmd, cwd=cwd, env=env, capture_output=True, text=True,
                           timeout=timeout)
    finally:
        _clear_ptx(cwd)
    wall = time.perf_counter() - t0
    if r.returncode != 0:
        raise RuntimeError(f"reference test_ycsb failed ({r.returncode}): {r.stderr[-2000:]}")
    out = {"wall_s": wall}
    for line in r.stdout.splitlines():
        m = _NUM.match(line.strip())
        if m:
            out[m.group(1)] = float(m.group(2))
    if "through" not in out:
        raise RuntimeError(f"no report in the reference's output: {r.stdout[-2000:]}")
    return out
