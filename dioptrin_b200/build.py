"""Builds libdioptrin_b200.so in-tree with nvcc for sm_100a.

    python -m dioptrin_b200.build

Each CUDA translation unit is compiled separately (dg_build.cu with
-fmad=false so the table builders do not fuse a*b+c, as the reference's Rust
does not) and linked into one shared library with the CUDA runtime linked
statically. The library exports only the C ABI declared in
include/dioptrin_gpu.h.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libdioptrin_b200.so")
OBJ = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "--expt-relaxed-constexpr",
          "-Xcompiler", "-fPIC,-ffp-contract=off,-fvisibility=hidden",
          "-I", os.path.join(ROOT, "include")]
SOURCES = {
    "dg_build.cu": ["-fmad=false"],
    "dg_scan.cu": [],
    "dg_gather.cu": [],
    "dg_api.cu": [],
    "dg_server.cu": [],
    "dg_bslz4.cu": [],
    "dg_multi.cu": [],
}


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build")
    return path


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(ROOT, "include", "dioptrin_gpu.h"))
    jobs = []
    objs = []
    for src, extra in SOURCES.items():
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _stale(o, [s] + headers):
            jobs.append([nvcc(), *ARCH, *COMMON, *extra, "-c", s, "-o", o])
    with cf.ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        for cmd, res in zip(jobs, ex.map(lambda c: subprocess.run(c, capture_output=True, text=True), jobs)):
            if verbose or res.returncode:
                sys.stderr.write(" ".join(cmd) + "\n" + res.stdout + res.stderr)
            if res.returncode:
                raise RuntimeError("nvcc failed on " + cmd[-3])
    if force or jobs or _stale(OUT, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", OUT, *objs, "-Xcompiler", "-fPIC"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if verbose or res.returncode:
            sys.stderr.write(" ".join(cmd) + "\n" + res.stdout + res.stderr)
        if res.returncode:
            raise RuntimeError("link of libdioptrin_b200.so failed")
    return OUT


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
