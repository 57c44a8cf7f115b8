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

CU_SOURCES = ["kernels.cu", "kernels_tma.cu", "solver.cu", "tuner.cu", "batch.cu", "noalloc.cu", "fft3d.cu"]
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


def ct_sizes():
    """Transform lengths listed in csrc/ct_sizes.h."""
    import re

    with open(os.path.join(CSRC, "ct_sizes.h")) as f:
        return [int(v) for v in re.findall(r"X\((\d+)\)", f.read())]


def tma_sizes():
    """Transform lengths listed in csrc/tma_sizes.h."""
    import re

    with open(os.path.join(CSRC, "tma_sizes.h")) as f:
        return [int(v) for v in re.findall(r"X\((\d+)\)", f.read())]


def _fused_sources():
    """One generated translation unit per TMA length: an explicit
    instantiation of the fused last-axis pass fused_tma_cls<N> (fused_tma.cuh)."""
    d = os.path.join(BUILD, "tma")
    os.makedirs(d, exist_ok=True)
    out = []
    for n in tma_sizes():
        path = os.path.join(d, f"fused_tma_{n}.cu")
        text = (f'#include "fused_tma.cuh"\nnamespace kwb {{\n'
                f'template cudaError_t fused_tma_cls<{n}>(const FusedTmaArgs&, const float2*, const SpecTables&,'
                f' cudaStream_t);\n}}\n')
        if not os.path.exists(path) or open(path).read() != text:
            with open(path, "w") as f:
                f.write(text)
        out.append(path)
    return out


def _ct_sources():
    """One generated translation unit per compile-time length: an explicit
    instantiation of CtKernels<N> (kernels_impl.cuh)."""
    d = os.path.join(BUILD, "ct")
    os.makedirs(d, exist_ok=True)
    out = []
    for n in ct_sizes():
        path = os.path.join(d, f"kernels_ct_{n}.cu")
        text = f'#include "kernels_impl.cuh"\nnamespace kwb {{\ntemplate struct CtKernels<{n}>;\n}}\n'
        if not os.path.exists(path) or open(path).read() != text:
            with open(path, "w") as f:
                f.write(text)
        out.append(path)
    return out


def build(force: bool = False, jobs: int = 0, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    jobs = jobs or os.cpu_count() or 4
    hdrs = _headers()
    jobs_list = []
    objs = []
    for s in _ct_sources() + _fused_sources():
        o = s[:-3] + ".o"
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            jobs_list.append([NVCC] + ARCH + CU_FLAGS + ["-c", s, "-o", o])
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
    ap.add_argument("--jobs", type=int, default=0, help="parallel compiles (0: one per CPU)")
    a = ap.parse_args()
    print(build(force=a.force, jobs=a.jobs, verbose=True))
