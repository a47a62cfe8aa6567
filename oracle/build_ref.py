"""Compile the reference's legacy translation (legacy/classicaldft.hpp of the
reference tree, read where it lies) behind the C-ABI shim
oracle/legacy_ref/legacy_ref.cpp into oracle/_ref/liblegacy_ref.so.

    python -m oracle.build_ref [REFERENCE_ROOT]

The reference's CMake build needs Armadillo, FFTW3, GSL and autodiff (none is
installed here); this one header needs none of them, so it is compiled
directly with g++ and an empty stand-in for its <armadillo> include.  Test
infrastructure only: the library never loads the result.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
LIB = os.path.join(OUT_DIR, "liblegacy_ref.so")
DEFAULT_REF = "/root/reference"


def build(reference_root: str = DEFAULT_REF, verbose: bool = False) -> str | None:
    """Build the shim; None (nothing done) when the reference tree is absent."""
    header = os.path.join(reference_root, "legacy", "classicaldft.hpp")
    if not os.path.exists(header):
        return None
    src = os.path.join(HERE, "legacy_ref", "legacy_ref.cpp")
    os.makedirs(OUT_DIR, exist_ok=True)
    if os.path.exists(LIB) and os.path.getmtime(LIB) > max(os.path.getmtime(src), os.path.getmtime(header)):
        return LIB
    cmd = ["g++", "-std=c++20", "-O2", "-fPIC", "-shared", "-I", os.path.join(HERE, "legacy_ref"), "-I",
           reference_root, src, "-o", LIB]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(sys.argv[1] if len(sys.argv) > 1 else DEFAULT_REF, verbose=True))
