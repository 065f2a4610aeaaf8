#!/usr/bin/env python3
"""Build libdgp.so (sm_100a) in-tree: dg-parallel_b200/lib/libdgp.so.

Every CUDA unit is compiled with ``nvcc -gencode arch=compute_100a,code=sm_100a``
in parallel; a unit is recompiled only when it or a header is newer than its
object.  ``python build.py [-j N] [--clean] [--ptxas-verbose]``.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "lib", "libdgp.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# FP32 division and square root by their fast approximations (the mixed form's
# right-hand side; FP64 arithmetic is not affected)
CUFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr",
           "--prec-div=false", "--prec-sqrt=false",
           "-I" + CSRC, "-I" + INCLUDE]


def headers() -> list[str]:
    return (glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) +
            glob.glob(os.path.join(INCLUDE, "*.h")))


def needs(obj: str, src: str, deps: list[str]) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(p) > t for p in [src] + deps)


def compile_one(src: str, verbose_ptxas: bool) -> tuple[str, int, str]:
    obj = os.path.join(OBJ, os.path.basename(src) + ".o")
    if src.endswith(".cu"):
        cmd = [NVCC] + ARCH + CUFLAGS + ["-c", src, "-o", obj]
        if verbose_ptxas:
            cmd[1:1] = ["-Xptxas", "-v"]
    else:
        cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-I" + CSRC, "-I" + INCLUDE, "-c", src, "-o", obj]
    p = subprocess.run(cmd, capture_output=True, text=True)
    return obj, p.returncode, p.stdout + p.stderr


def build(jobs: int = 0, clean: bool = False, verbose_ptxas: bool = False, quiet: bool = False) -> str:
    if clean and os.path.isdir(OBJ):
        shutil.rmtree(OBJ)
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    deps = headers()
    todo = [s for s in srcs if needs(os.path.join(OBJ, os.path.basename(s) + ".o"), s, deps)]
    jobs = jobs or min(len(todo) or 1, os.cpu_count() or 4)
    failed = []
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        for obj, rc, log in ex.map(lambda s: compile_one(s, verbose_ptxas), todo):
            if rc != 0:
                failed.append((obj, log))
            elif log.strip() and (verbose_ptxas or not quiet):
                sys.stderr.write(log)
    if failed:
        for obj, log in failed:
            sys.stderr.write(f"--- {obj}\n{log}\n")
        raise RuntimeError(f"{len(failed)} unit(s) failed to compile")
    objs = [os.path.join(OBJ, os.path.basename(s) + ".o") for s in srcs]
    if todo or not os.path.exists(LIB):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart_static", "-lrt", "-ldl", "-lpthread"]
        p = subprocess.run(cmd, capture_output=True, text=True)
        if p.returncode != 0:
            raise RuntimeError("link failed:\n" + p.stdout + p.stderr)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("-j", type=int, default=0)
    ap.add_argument("--clean", action="store_true")
    ap.add_argument("--ptxas-verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.j, a.clean, a.ptxas_verbose))
