"""Build the engine's shared library in-tree for sm_100a.

    python -m classicaldft_b200.build            # -> classicaldft_b200/libcdft_b200.so

nvcc compiles every source with -gencode arch=compute_100a,code=sm_100a and
links cuFFT; objects go to classicaldft_b200/_build/.  A source is rebuilt
only when it (or a header) is newer than its object.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libcdft_b200.so")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc") if os.path.exists(os.path.join(CUDA_HOME, "bin", "nvcc")) else "nvcc"

SOURCES = ["engine.cu", "fused.cu", "drivers.cu", "lanczos.cu", "host_stream.cu", "capi.cu", "noalloc.cu", "bulk.cu",
           "lattice.cu", "physics.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++20", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "--expt-relaxed-constexpr", "-I", CSRC, "-I", os.path.join(ROOT, "include")]


def _headers():
    out = []
    for d in (CSRC, os.path.join(ROOT, "include")):
        for f in os.listdir(d):
            if f.endswith((".cuh", ".hpp", ".h")):
                out.append(os.path.join(d, f))
    return out


def _stale(obj, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def _deps(src, obj, headers):
    """The headers a source includes, from the dependency file nvcc / g++
    wrote beside its object (-MD); every header when there is none yet."""
    dfile = obj + ".d"
    if not os.path.exists(dfile):
        return headers
    with open(dfile) as f:
        text = f.read().replace("\\\n", " ")
    out = []
    for tok in text.split(":", 1)[-1].split():
        if os.path.exists(tok) and os.path.abspath(tok).startswith(ROOT):
            out.append(tok)
    return out or headers


def build(verbose: bool = False, extra=None) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = _headers()
    objs, cmds = [], []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if not _stale(obj, [path] + _deps(path, obj, headers)):
            continue
        cmd = [NVCC] + ARCH + FLAGS + (extra or []) + ["-MD", "-MF", obj + ".d", "-c", path, "-o", obj]
        if src.endswith(".cpp"):
            cmd = ["g++", "-O3", "-std=c++17", "-fPIC", "-fvisibility=hidden", "-I", CSRC, "-I",
                   os.path.join(ROOT, "include"), "-I", os.path.join(CUDA_HOME, "include"), "-MD", "-MF",
                   obj + ".d", "-c", path, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        cmds.append(cmd)
    # translation units compile in parallel
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        for f in [ex.submit(subprocess.run, c, check=True) for c in cmds]:
            f.result()
    if _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + [
            "-L", os.path.join(CUDA_HOME, "lib64"), "-lcufft", "-lcudart",
            "-Xlinker", "-rpath," + os.path.join(CUDA_HOME, "lib64")]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print(LIB)
