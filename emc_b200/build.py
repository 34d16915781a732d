"""Builds libemc_b200.so in-tree for sm_100a with nvcc.

    python -m emc_b200.build          # incremental
    python -m emc_b200.build --force  # full rebuild
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
OUT = os.path.join(HERE, "libemc_b200.so")
OBJDIR = os.path.join(HERE, "_build")
SOURCES = ["host.cpp", "kernels_fp32.cu", "kernels_tc.cu", "context.cu", "legacy.cu", "noalloc.cu",
           "net.cu", "proposal.cu"]
HEADERS = ["voxel.h", "kernels.cuh", "tc.cuh", "tile.cuh", "proposal.cuh", "fixed.cuh"]
PUBLIC = [os.path.join(REPO, "include", h) for h in ("emc.h", "emc_b200.h")]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
HOST = ["-Xcompiler", "-fPIC,-fopenmp,-ffp-contract=off,-O3"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr"] + ARCH + HOST


def _nvcc():
    for cand in ("/usr/local/cuda/bin/nvcc", "nvcc"):
        if os.path.sep not in cand or os.path.isfile(cand):
            return cand
    return "nvcc"


def _stale(target, deps):
    if not os.path.isfile(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.isfile(d))


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJDIR, exist_ok=True)
    csrc = os.path.join(HERE, "csrc")
    headers = [os.path.join(csrc, h) for h in HEADERS] + PUBLIC
    jobs = []
    objs = []
    for s in SOURCES:
        src = os.path.join(csrc, s)
        obj = os.path.join(OBJDIR, s + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            jobs.append([_nvcc()] + NVCC_FLAGS + ["-c", src, "-o", obj])
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        for cmd, res in zip(jobs, ex.map(lambda c: subprocess.run(c, capture_output=True, text=True), jobs)):
            if verbose or res.returncode != 0:
                sys.stderr.write(" ".join(cmd) + "\n" + res.stdout + res.stderr)
            if res.returncode != 0:
                raise RuntimeError(f"nvcc failed on {cmd[-3]}")
    if force or jobs or _stale(OUT, objs):
        cmd = [_nvcc(), "-shared"] + ARCH + ["-o", OUT] + objs + ["-Xcompiler", "-fopenmp", "-lgomp"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            sys.stderr.write(" ".join(cmd) + "\n" + res.stdout + res.stderr)
            raise RuntimeError("link of libemc_b200.so failed")
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
