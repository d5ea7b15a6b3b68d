"""Build libplastimatch_b200.so in-tree with nvcc for sm_100a.

    python -m plastimatch_b200.build          # or build() from Python

Every .cu under plastimatch_b200/csrc is compiled separately (in parallel)
with  -gencode arch=compute_100a,code=sm_100a -lineinfo -O3  and linked into
plastimatch_b200/libplastimatch_b200.so next to this file, so the library
travels with the source tree.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libplastimatch_b200.so")
ROOT = os.path.dirname(HERE)

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
              "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]
# per-source flags: the optimiser's device controller rounds as its host
# counterpart does (no multiply-add contraction)
FILE_FLAGS = {"lbfgs_graph.cu": ["-fmad=false"]}


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc",
                 shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def host_cxx() -> str:
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def build(verbose: bool = False, force: bool = False, extra_flags=()) -> str:
    os.makedirs(BUILD, exist_ok=True)
    nvcc = nvcc_path()
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    headers = (glob.glob(os.path.join(CSRC, "*.cuh"))
               + glob.glob(os.path.join(ROOT, "include", "*.h")))
    objs = []
    jobs = []
    for src in sources:
        obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        if force or not _newer(obj, [src] + headers):
            cmd = ([nvcc, "-ccbin", host_cxx()] + ARCH + NVCC_FLAGS
                   + FILE_FLAGS.get(os.path.basename(src), [])
                   + list(extra_flags) + ["-I", CSRC, "-I",
                                          os.path.join(ROOT, "include"),
                                          "-c", src, "-o", obj])
            jobs.append(cmd)

    def run(cmd):
        p = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, p

    with ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        for cmd, p in ex.map(run, jobs):
            if verbose or p.returncode != 0:
                sys.stderr.write(" ".join(cmd[-3:]) + "\n" + p.stdout + p.stderr)
            if p.returncode != 0:
                raise RuntimeError(f"nvcc failed on {cmd[-3]}")
    if force or jobs or not _newer(LIB, objs):
        cmd = ([nvcc, "-ccbin", host_cxx()] + ARCH
               + ["-shared", "-o", LIB] + objs + ["-lcuda"])
        p = subprocess.run(cmd, capture_output=True, text=True)
        if p.returncode != 0:
            sys.stderr.write(p.stdout + p.stderr)
            raise RuntimeError("link failed")
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(LIB)
