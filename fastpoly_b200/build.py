"""Builds the in-tree CUDA library fastpoly_b200/libfpx_b200.so for sm_100a,
and the CPython helper fastpoly_b200/_fpx_jobs (batch job records).

    python -m fastpoly_b200.build [--force]

nvcc compiles the kernels (-gencode arch=compute_100a,code=sm_100a -lineinfo),
g++ the C++20 host engine and the C ABI, linked against the static CUDA
runtime so the library carries no runtime-path dependency.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libfpx_b200.so")
INCLUDE = os.path.join(ROOT, "include")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CU_SOURCES = ["kernels.cu", "noalloc.cu", "peaks.cu"]
CPP_SOURCES = ["engine.cpp", "batch.cpp", "serve.cpp", "tune.cpp", "api.cpp"]
HEADERS = ["field.cuh", "ntt_core.cuh", "ntt_fast.cuh", "kernels.h", "engine.h"]


def _sources():
    out = [os.path.join(CSRC, s) for s in CU_SOURCES + CPP_SOURCES + HEADERS]
    out.append(os.path.join(INCLUDE, "fpx_b200.h"))
    return out


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(s) > t for s in _sources() if os.path.exists(s))


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd)
    if r.returncode != 0:
        raise RuntimeError(f"build step failed with status {r.returncode}: {cmd[0]} {cmd[-1]}")


def _object_stale(src: str, obj: str, headers: list) -> bool:
    """An object is rebuilt when it is missing or older than its source or any
    header of the library (headers are shared, so any change rebuilds all)."""
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return os.path.getmtime(src) > t or any(os.path.getmtime(h) > t for h in headers if os.path.exists(h))


PYJOBS_SRC = os.path.join(CSRC, "pyjobs.c")
PYJOBS = os.path.join(HERE, "_fpx_jobs" + (sysconfig.get_config_var("EXT_SUFFIX") or ".so"))


def build_pyjobs(force: bool = False, verbose: bool = False) -> str:
    """The CPython extension that fills batch job records (plain C, no CUDA)."""
    deps = [PYJOBS_SRC, os.path.join(INCLUDE, "fpx_b200.h")]
    if not force and os.path.exists(PYJOBS) and all(os.path.getmtime(d) <= os.path.getmtime(PYJOBS) for d in deps):
        return PYJOBS
    cc = os.environ.get("CC", shutil.which("gcc") or "cc")
    tmp = PYJOBS + ".tmp"
    _run([cc, "-O2", "-fPIC", "-shared", "-Wall", "-I" + sysconfig.get_paths()["include"], "-I" + INCLUDE,
          PYJOBS_SRC, "-o", tmp], verbose)
    os.replace(tmp, PYJOBS)
    return PYJOBS


def build(force: bool = False, verbose: bool = False) -> str:
    build_pyjobs(force, verbose)
    if not force and not _stale():
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "fpx_b200.h")]
    cxx = os.environ.get("CXX", shutil.which("g++") or "g++")
    jobs, objs = [], []
    for s in CU_SOURCES:
        src, o = os.path.join(CSRC, s), os.path.join(BUILD, s + ".o")
        objs.append(o)
        if force or _object_stale(src, o, headers):
            jobs.append([NVCC, "-std=c++17", "-O3", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC", "-I" + CSRC,
                         "-I" + INCLUDE, "-c", src, "-o", o])
    for s in CPP_SOURCES:
        src, o = os.path.join(CSRC, s), os.path.join(BUILD, s + ".o")
        objs.append(o)
        if force or _object_stale(src, o, headers):
            jobs.append([cxx, "-std=c++20", "-O2", "-fPIC", "-Wall", "-I" + CSRC, "-I" + INCLUDE,
                         "-I" + os.path.join(CUDA_HOME, "include"), "-c", src, "-o", o])
    # the translation units compile in parallel (the kernels dominate)
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        for f in [ex.submit(_run, j, verbose) for j in jobs]:
            f.result()
    tmp = LIB + ".tmp"
    # --exclude-libs: symbols of static archives (the CUDA runtime, and the C++
    # runtime where the toolchain links it statically) stay private, so a host
    # process holding its own copies (Python with libstdc++.so) cannot interpose
    # them half-way.
    _run([cxx, "-shared", "-o", tmp, *objs, "-L" + os.path.join(CUDA_HOME, "lib64"), "-lcudart_static", "-ldl",
          "-lrt", "-pthread", "-Wl,--exclude-libs,ALL"], verbose)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
