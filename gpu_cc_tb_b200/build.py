"""Build the engine's native artefacts in-tree.

Outputs (git-ignored, shipped with the source tree):
  gpu_cc_tb_b200/lib/libgcctb.so   the C-ABI library (include/gcc_engine.h)
  gpu_cc_tb_b200/bin/test_ycsb     drop-in for gCCTB's test_ycsb CLI
  gpu_cc_tb_b200/bin/gen_ycsb      drop-in for gCCTB's gen_ycsb CLI

Every CUDA translation unit is compiled for sm_100a only. Objects are cached
in gpu_cc_tb_b200/_build and rebuilt when a source or header is newer.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OBJ = PKG / "_build"
LIB = PKG / "lib"
BIN = PKG / "bin"
INCLUDE = ROOT / "include"

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I", str(INCLUDE)]
CXXFLAGS = ["-O2", "-std=c++17", "-fPIC", "-I", str(INCLUDE)]

CU_UNITS = ["engine", "cc_tpl", "cc_to", "cc_mvcc", "cc_silo", "cc_tictoc", "cc_ordered", "cc_var", "cc_var_slow", "sched",
            "noalloc", "calib"]
CXX_UNITS = ["gen", "orderentry"]
HEADERS = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(INCLUDE.glob("*.h"))

LIBRARY = LIB / "libgcctb.so"


def _newest(paths):
    return max((p.stat().st_mtime for p in paths if p.exists()), default=0.0)


def _stale(out: Path, deps) -> bool:
    return not out.exists() or out.stat().st_mtime < _newest(deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build step failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r


def build(verbose: bool = False, jobs: int | None = None) -> Path:
    OBJ.mkdir(exist_ok=True)
    LIB.mkdir(exist_ok=True)
    BIN.mkdir(exist_ok=True)
    cmds = []
    objs = []
    for u in CU_UNITS:
        src, obj = CSRC / f"{u}.cu", OBJ / f"{u}.o"
        objs.append(obj)
        if _stale(obj, [src, *HEADERS]):
            cmds.append([NVCC, *ARCH, *CUFLAGS, "-c", str(src), "-o", str(obj)])
    for u in CXX_UNITS:
        src, obj = CSRC / f"{u}.cpp", OBJ / f"{u}.o"
        objs.append(obj)
        if _stale(obj, [src, *HEADERS]):
            cmds.append(["g++", *CXXFLAGS, "-c", str(src), "-o", str(obj)])
    jobs = jobs or max(1, min(len(cmds), os.cpu_count() or 1))
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        for r in ex.map(_run, cmds):
            if verbose and r.stderr:
                print(r.stderr, file=sys.stderr)
    if _stale(LIBRARY, objs):
        _run([NVCC, *ARCH, "-shared", "-Xcompiler", "-fPIC", "-o", str(LIBRARY),
              *map(str, objs), "-lpthread"])
    for tool in ("test_ycsb", "gen_ycsb"):
        src, exe = CSRC / f"{tool}_main.cpp", BIN / tool
        if src.exists() and _stale(exe, [src, LIBRARY, *HEADERS]):
            _run(["g++", *CXXFLAGS, str(src), "-o", str(exe), f"-L{LIB}", "-lgcctb",
                  f"-Wl,-rpath,$ORIGIN/../lib", "-lpthread"])
    return LIBRARY


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
