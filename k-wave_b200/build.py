"""Build the solver library and command-line binary in-tree with nvcc.

Outputs (next to this file):
  libkwave_b200.so      -- the C-ABI library declared in include/kwave_b200.h
  kspaceFirstOrder-B200 -- the drop-in command-line binary

Usage: python k-wave_b200/build.py [--force] [--jobs N]
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "libkwave_b200.so")
EXE = os.path.join(HERE, "kspaceFirstOrder-B200")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-O3",
            "-I" + INCLUDE, "-I" + CSRC]
CXX_FLAGS = ["-std=c++17", "-O3", "-fPIC", "-I" + INCLUDE, "-I" + CSRC, "-I/usr/local/cuda/include"]

CU_SOURCES = ["kernels.cu", "kernels_tma.cu", "solver.cu", "noalloc.cu"]
CXX_SOURCES = ["hdf5_lite.cpp", "io.cpp"]


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))] + [
        os.path.join(INCLUDE, "kwave_b200.h")]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: " + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r


def build(force: bool = False, jobs: int = 4, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hdrs = _headers()
    jobs_list = []
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            jobs_list.append([NVCC] + ARCH + CU_FLAGS + ["-c", s, "-o", o])
    for src in CXX_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            jobs_list.append(["g++"] + CXX_FLAGS + ["-c", s, "-o", o])
    with ThreadPoolExecutor(max_workers=max(1, jobs)) as ex:
        for r in ex.map(_run, jobs_list):
            if verbose:
                sys.stdout.write(r.stdout + r.stderr)
    if force or _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lz", "-lcudart"])
    main_src = os.path.join(CSRC, "main.cpp")
    if force or _stale(EXE, [main_src, LIB]):
        _run(["g++"] + CXX_FLAGS + [main_src, "-o", EXE, "-L" + HERE, "-lkwave_b200",
                                    "-Wl,-rpath,$ORIGIN"])
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=4)
    a = ap.parse_args()
    print(build(force=a.force, jobs=a.jobs, verbose=True))
