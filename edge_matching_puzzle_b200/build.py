"""Builds the native library of edge_matching_puzzle_b200 in-tree.

    python -m edge_matching_puzzle_b200.build [--force] [--jobs N]

Outputs (git-ignored, travel with the source tree):
  edge_matching_puzzle_b200/libemp_b200.so       C ABI of include/emp_b200.h (CUDA, sm_100a)
  edge_matching_puzzle_b200/edge_matching_puzzle host CLI mirroring the reference's main
Every .cu file is compiled with ``-gencode arch=compute_100a,code=sm_100a -lineinfo``;
host C++ files with g++ -O3.  Objects go to edge_matching_puzzle_b200/_build/.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
HOST = os.path.join(CSRC, "host")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libemp_b200.so")
CLI = os.path.join(HERE, "edge_matching_puzzle")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
INCLUDES = ["-I" + os.path.join(ROOT, "include"), "-I" + CSRC]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _sources(directory, exts):
    return sorted(os.path.join(directory, f) for f in os.listdir(directory) if f.endswith(exts))


def _headers():
    hs = [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))]
    hs += [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    if os.path.isdir(HOST):
        hs += [os.path.join(HOST, f) for f in os.listdir(HOST) if f.endswith(".h")]
    return hs


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src, obj, headers, verbose):
    if src.endswith(".cu"):
        cmd = [nvcc(), "-c", src, "-o", obj, "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-lineinfo",
               "--expt-relaxed-constexpr", *ARCH, *INCLUDES]
        if verbose:
            cmd += ["-Xptxas", "-v"]
    else:
        cmd = ["g++", "-c", src, "-o", obj, "-O3", "-std=c++17", "-fPIC", "-Wall", "-Wextra",
               "-I/usr/local/cuda/include", *INCLUDES]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r.stderr


def build(force: bool = False, jobs: int = 0, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = _headers()
    lib_srcs = _sources(CSRC, (".cu", ".cpp"))
    objs = []
    todo = []
    for src in lib_srcs:
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            todo.append((src, obj))
    logs = []
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 1)) as ex:
        for out in ex.map(lambda so: _compile(so[0], so[1], headers, verbose), todo):
            logs.append(out)
    if force or todo or _stale(LIB, objs):
        cmd = [nvcc(), "-shared", "-o", LIB, *objs, *ARCH, "-lcudart", "-Xlinker", "-rpath=/usr/local/cuda/lib64"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if os.path.isdir(HOST):
        host_srcs = _sources(HOST, (".cpp",))
        if host_srcs and (force or _stale(CLI, host_srcs + headers + [LIB])):
            cmd = ["g++", "-O3", "-std=c++17", "-o", CLI, *host_srcs, *INCLUDES, "-I" + HOST,
                   "-L" + HERE, "-lemp_b200", "-Wl,-rpath,$ORIGIN", "-lpthread"]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"CLI build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return "\n".join(l for l in logs if l)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=0)
    ap.add_argument("--verbose", action="store_true", help="print ptxas register/spill report")
    a = ap.parse_args()
    out = build(a.force, a.jobs, a.verbose)
    if out:
        print(out)
    print(LIB)


if __name__ == "__main__":
    sys.exit(main())
