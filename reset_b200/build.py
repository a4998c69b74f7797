"""Builds libreset.so (all CUDA sources under csrc/) for sm_100a with nvcc.

The shared library is built in-tree (reset_b200/libreset.so) so it travels
with the repository snapshot; objects go to reset_b200/_build/.  Rebuilds
only what changed (source or header newer than its object).

    python -m reset_b200.build [--force] [--ptxas-v]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libreset.so")
HOST = os.path.join(PKG, "host")
BIN = os.path.join(PKG, "bin")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                  "-I", INCLUDE, "-I", CSRC, "--expt-relaxed-constexpr"]


def nvcc() -> str:
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(p):
        raise RuntimeError("nvcc not found")
    return p


def _headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h"))


def _stale(obj: str, deps) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, ptxas_verbose: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    hdrs = _headers()
    jobs = []
    for s in srcs:
        obj = os.path.join(BUILD, os.path.basename(s)[:-3] + ".o")
        if force or _stale(obj, [s] + hdrs):
            cmd = [nvcc()] + NVFLAGS + (["-Xptxas", "-v"] if ptxas_verbose else []) + \
                ["-c", s, "-o", obj]
            jobs.append((s, cmd))
    objs = [os.path.join(BUILD, os.path.basename(s)[:-3] + ".o") for s in srcs]

    def run(job):
        s, cmd = job
        r = subprocess.run(cmd, capture_output=True, text=True)
        return s, r

    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            for s, r in ex.map(run, jobs):
                if r.returncode != 0:
                    sys.stderr.write(r.stdout + r.stderr)
                    raise RuntimeError(f"nvcc failed on {os.path.basename(s)}")
                if verbose or ptxas_verbose:
                    sys.stderr.write(r.stdout + r.stderr)
    if force or jobs or _stale(LIB, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link of libreset.so failed")
    build_host_tools(force)
    return LIB


def build_host_tools(force: bool = False):
    """C++ drop-in drivers (host/*.cpp) linked against libreset.so."""
    os.makedirs(BIN, exist_ok=True)
    cxx = shutil.which("g++") or "g++"
    hdrs = [os.path.join(INCLUDE, "reset.h"), os.path.join(INCLUDE, "reset.hpp")]
    for src in sorted(glob.glob(os.path.join(HOST, "*.cpp"))):
        exe = os.path.join(BIN, os.path.basename(src)[:-4])
        if not force and not _stale(exe, [src, LIB] + hdrs):
            continue
        cmd = [cxx, "-O2", "-std=c++17", "-I", INCLUDE, "-I", os.path.join(CUDA_HOME, "include"),
               src, "-o", exe, "-L", PKG, "-lreset", "-L", os.path.join(CUDA_HOME, "lib64"),
               "-lcudart", "-Wl,-rpath,$ORIGIN/..", "-Wl,-rpath," + os.path.join(CUDA_HOME, "lib64")]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"build of {os.path.basename(exe)} failed")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, ptxas_verbose=a.ptxas_v, verbose=True))


if __name__ == "__main__":
    main()
