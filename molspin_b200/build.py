"""In-tree build of the msgpu shared library (CUDA for sm_100a + host C++).

The library is built next to this file as ``libmsgpu.so`` so that it travels
with the source tree; nothing is installed into site-packages.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "libmsgpu.so")

SOURCES = ["msgpu_api.cu", "msgpu_batch.cu", "msgpu_dense.cu", "msgpu_host.cpp"]
HEADERS = ["msgpu_device.cuh", "msgpu_kernels.cuh", "msgpu_resident.cuh", "msgpu_batch.cuh", "msgpu_dense.h", "msgpu_philox.h",
           "msgpu_fused.cuh", "msgpu_spmm_tc.cuh", "msgpu_spmm_tm.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
    "--expt-relaxed-constexpr",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, extra_flags: list[str] | None = None) -> str:
    """Compile libmsgpu.so if any source changed; returns its path."""
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    deps = srcs + [os.path.join(CSRC, h) for h in HEADERS] + [
        os.path.join(INCLUDE, "msgpu.h"), os.path.join(INCLUDE, "msgpu_host.h")]
    if not force and not _stale(LIB, deps):
        return LIB
    objs = []
    for s in srcs:
        obj = os.path.join(CSRC, os.path.basename(s) + ".o")
        cmd = [_nvcc(), *NVCC_FLAGS, *(extra_flags or []), "-I", INCLUDE, "-I", CSRC, "-c", s, "-o", obj]
        if s.endswith(".cpp"):
            cmd = ["g++", "-O3", "-std=c++17", "-fPIC", "-I", INCLUDE, "-I", CSRC, "-c", s, "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    link = [_nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", LIB, *objs, "-lcudart"]
    if verbose:
        print(" ".join(link), file=sys.stderr)
    subprocess.run(link, check=True)
    for o in objs:
        os.remove(o)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
