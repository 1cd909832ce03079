"""Builds the native library libsubfv_b200.so in-tree with nvcc for sm_100a.

Every .cu/.cpp under subfv_b200/csrc goes into one shared library exposing the C-ABI
of include/subfv.h. The plain-FP64 kernels need --fmad=false (no FMA contraction) to
evaluate expressions exactly as the reference does.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
OUT_DIR = PKG / "_build"
LIB = OUT_DIR / "libsubfv_b200.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC,-O2",
         "-Xptxas", "-O3", "--expt-relaxed-constexpr"]


def sources():
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = sources() + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + [PKG.parent / "include" / "subfv.h"]
    return any(p.stat().st_mtime > t for p in deps)


def _headers():
    return list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + [PKG.parent / "include" / "subfv.h"]


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not _stale():
        return LIB
    OUT_DIR.mkdir(exist_ok=True)
    newest_header = max(p.stat().st_mtime for p in _headers())
    jobs = []
    for src in sources():
        obj = OUT_DIR / (src.name + ".o")
        fresh = obj.exists() and obj.stat().st_mtime > max(src.stat().st_mtime, newest_header)
        cmd = [NVCC, *ARCH, *FLAGS, "-I", str(PKG.parent / "include"), "-c", str(src), "-o", str(obj)]
        jobs.append((cmd, obj, force or not fresh))

    def run(job):
        cmd, obj, todo = job
        if todo:
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
        return str(obj)

    with ThreadPoolExecutor(max_workers=max(1, min(8, os.cpu_count() or 1))) as ex:
        objs = list(ex.map(run, jobs))
    tmp = LIB.with_suffix(".so.tmp")
    subprocess.run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", str(tmp), *objs], check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
