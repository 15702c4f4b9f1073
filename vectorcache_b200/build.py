"""Build the in-tree CUDA library vectorcache_b200/libvectorcache_b200.so.

nvcc compiles every kernel for sm_100a only. Host and device code are built
without floating-point contraction (-fmad=false, -ffp-contract=off): every
fused multiply-add the arithmetic needs is written explicitly, so the results
do not depend on compiler choices.

Usage: python -m vectorcache_b200.build [--force]
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB = PKG / "libvectorcache_b200.so"
SOURCES = ["tq_host_math.cpp", "tq_formats.cpp", "tq_encode.cu", "tq_query.cu", "tq_scan.cu", "tq_bigdim.cu",
           "tq_bucket.cu", "tq_bucketed.cu", "tq_probe.cu", "tq_server.cu", "tq_multi.cu",
           "tq_rescore.cu", "tq_index.cu"]
HEADERS = ["tq_host_math.h", "tq_kernels.h", "tq_device.cuh", "tq_abi.h", "tq_index_impl.h", "tq_bucket.h",
           "tq_probe.h", "tq_serving_hooks.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = [CSRC / s for s in SOURCES + HEADERS] + [PKG.parent / "include" / "vectorcache_b200.h", Path(__file__)]
    return any(p.stat().st_mtime > t for p in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not _stale():
        return LIB
    out_dir = PKG / "_build"
    out_dir.mkdir(exist_ok=True)
    objs = []
    common = [
        "-O3", "-std=c++17", "-lineinfo", "-fmad=false",
        "-Xcompiler", "-fPIC,-ffp-contract=off",
        "-I", str(PKG.parent / "include"),
    ]
    cmds = []
    for src in SOURCES:
        obj = out_dir / (Path(src).stem + ".o")
        cmds.append([nvcc(), *ARCH, *common, "-c", str(CSRC / src), "-o", str(obj)])
        objs.append(str(obj))
    with ThreadPoolExecutor(max_workers=len(cmds)) as pool:
        for cmd in cmds:
            if verbose:
                print(" ".join(cmd), flush=True)
        for fut in [pool.submit(subprocess.run, cmd, check=True) for cmd in cmds]:
            fut.result()
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *objs, "-Xcompiler", "-fPIC"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
