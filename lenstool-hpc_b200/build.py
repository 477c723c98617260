"""Build liblt_b200.so (the CUDA kernels and the C ABI) in-tree for sm_100a with nvcc.

    python lenstool-hpc_b200/build.py [--verbose] [--ptxas-info]

Objects go to lenstool-hpc_b200/_build/, the library to lenstool-hpc_b200/liblt_b200.so.
Only changed sources are recompiled (their headers are tracked coarsely: any header
change rebuilds everything).
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import pathlib
import shutil
import subprocess
import sys

PKG = pathlib.Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "liblt_b200.so"
INCLUDE = PKG.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-ffp-contract=off", "-Xcompiler", "-Wall", "-I", str(INCLUDE)]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and pathlib.Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def headers():
    return sorted(list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h")))


def _compile(src: pathlib.Path, obj: pathlib.Path, extra, verbose: bool):
    cmd = [nvcc()] + ARCH + NVCC_FLAGS + extra + ["-c", str(src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    return src, r


def build(verbose: bool = False, ptxas_info: bool = False, force: bool = False) -> pathlib.Path:
    BUILD.mkdir(exist_ok=True)
    hdr_mtime = max((h.stat().st_mtime for h in headers()), default=0.)
    jobs = []
    objs = []
    for src in sources():
        obj = BUILD / (src.name + ".o")
        objs.append(obj)
        if force or ptxas_info or not obj.exists() or obj.stat().st_mtime < max(src.stat().st_mtime, hdr_mtime):
            jobs.append((src, obj))
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    failed = []
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        for src, r in ex.map(lambda j: _compile(j[0], j[1], extra, verbose), jobs):
            if r.returncode != 0 or ptxas_info:
                sys.stderr.write(r.stderr)
            if r.returncode != 0:
                failed.append(src.name)
    if failed:
        raise RuntimeError(f"nvcc failed for {failed}")
    if jobs or not LIB.exists():
        cmd = [nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", str(LIB)] + [str(o) for o in objs]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stderr)
            raise RuntimeError("link failed")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(a.verbose, a.ptxas_info, a.force))
