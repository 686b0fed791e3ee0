"""Build libb200qz.so (sm_100a) in-tree with nvcc.

    python gevp-pdhgeqz_b200/build.py [--verbose-ptxas]

Every translation unit is compiled with
``-gencode arch=compute_100a,code=sm_100a -O3 -lineinfo`` and linked into
``gevp-pdhgeqz_b200/libb200qz.so``.  Objects go to
``gevp-pdhgeqz_b200/_build/``.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libb200qz.so")
SOURCES = ["kernels.cu", "batched.cu", "policy.cu", "ozaki.cu", "balance.cu", "reorder.cu", "hessred.cu", "capi.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _newer(src_list, target):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in src_list)


def build(verbose_ptxas: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(HERE, "..", "include", "b200qz.h"))
    flags = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"] + ARCH
    if verbose_ptxas:
        flags += ["-Xptxas", "-v"]
    objs = []
    jobs = []
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, s.replace(".cu", ".o"))
        objs.append(obj)
        if force or verbose_ptxas or _newer([src] + headers, obj):
            jobs.append([nvcc(), "-c", src, "-o", obj] + flags)
    with cf.ThreadPoolExecutor(max_workers=max(1, len(jobs))) as ex:
        for cmd, res in zip(jobs, ex.map(lambda c: subprocess.run(c, capture_output=True, text=True), jobs)):
            if res.returncode != 0 or verbose_ptxas:
                sys.stderr.write(res.stdout + res.stderr)
            if res.returncode != 0:
                raise RuntimeError("nvcc failed: " + " ".join(cmd))
    if force or jobs or _newer(objs, LIB):
        cmd = [nvcc(), "-shared", "-o", LIB] + objs + ARCH + ["-lcudart"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            sys.stderr.write(res.stdout + res.stderr)
            raise RuntimeError("link failed")
    return LIB


if __name__ == "__main__":
    print(build(verbose_ptxas="--verbose-ptxas" in sys.argv, force="--force" in sys.argv))
