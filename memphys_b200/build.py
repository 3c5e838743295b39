"""Build libmemphys_cuda.so (sm_100a) in-tree with nvcc.

Every ``csrc/*.cu`` file is compiled to an object under ``_build/`` (in
parallel, rebuilt when it or any header is newer than its object) and linked
into ``memphys_b200/libmemphys_cuda.so``.  The library depends only on the CUDA
runtime; it exports the C ABI declared in ``include/memphys.h``.

    python -m memphys_b200.build [--force] [--verbose]
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(HERE, "libmemphys_cuda.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O2",
                     "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include")]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libmemphys_cuda.so")


def _headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(ROOT, "include", "*.h"))


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    newest_hdr = max((os.path.getmtime(h) for h in _headers()), default=0.0)
    cc = nvcc()
    jobs = []
    objs = []
    for s in srcs:
        o = os.path.join(BUILD, os.path.basename(s)[:-3] + ".o")
        objs.append(o)
        if force or not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), newest_hdr):
            jobs.append((s, o))

    def compile_one(job):
        s, o = job
        cmd = [cc] + NVCC_FLAGS + ["-c", s, "-o", o]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {os.path.basename(s)}:\n{r.stderr}")
        return r.stderr

    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
            for out in ex.map(compile_one, jobs):
                if verbose and out:
                    print(out)
    if force or jobs or not os.path.exists(LIB):
        cmd = [cc] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}")
    build_host_driver(force)
    return LIB


DRIVER_SRC = os.path.join(HERE, "host", "cavity_driver.cpp")
DRIVER = os.path.join(HERE, "host", "cavity_driver")


def build_host_driver(force: bool = False) -> str:
    """The C++ example driver over the C ABI (host code only: g++ and the .so)."""
    deps = [DRIVER_SRC, os.path.join(HERE, "host", "memphys.hpp"), LIB]
    if force or not os.path.exists(DRIVER) or os.path.getmtime(DRIVER) < max(
            os.path.getmtime(d) for d in deps):
        cmd = ["g++", "-O2", "-std=c++17", "-Wall", DRIVER_SRC, "-o", DRIVER,
               "-L" + HERE, "-lmemphys_cuda", "-Wl,-rpath,$ORIGIN/.."]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"host driver build failed:\n{r.stderr}")
    return DRIVER


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="--verbose" in sys.argv))
