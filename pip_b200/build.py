"""In-tree build of the CUDA library (pip_b200/libpipgpu.so) for sm_100a.

Each ``.cu`` under ``csrc/`` is compiled with nvcc to an object and the objects are
linked into one shared library whose exported symbols are the ``extern "C"`` functions
of include/pip_gpu.h.  Per-file flag overrides (the FMA-free FP64 flavour) live in
``EXTRA_FLAGS``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from typing import List

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libpipgpu.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
          "-Xcompiler", "-Wno-unknown-pragmas", "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]
EXTRA_FLAGS = {
    "pip_fp64_exact.cu": ["-fmad=false"],
    "pip_mixed.cu": ["-ftz=true", "-prec-div=false", "-prec-sqrt=false"],
    "pip_ensemble.cu": ["-ftz=true", "-prec-div=false", "-prec-sqrt=false"],
}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources() -> List[str]:
    return sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))


def _deps_mtime() -> float:
    return max(os.path.getmtime(os.path.join(CSRC, f)) for f in os.listdir(CSRC)
               if f.endswith((".cu", ".cuh", ".h")))


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    """Compile every csrc/*.cu for sm_100a and link libpipgpu.so; returns its path."""
    inc = os.path.join(os.path.dirname(HERE), "include")
    newest = max([_deps_mtime(), os.path.getmtime(os.path.abspath(__file__))] +
                 [os.path.getmtime(os.path.join(inc, f)) for f in os.listdir(inc)])
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= newest:
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    objs = []
    for src in sources():
        obj = os.path.join(BUILD, src[:-3] + ".o")
        cmd = [nvcc()] + ARCH + COMMON + EXTRA_FLAGS.get(src, [])
        if ptxas_info:
            cmd += ["-Xptxas", "-v"]
        cmd += ["-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [nvcc()] + ARCH + ["-shared", "-o", tmp] + objs
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_info="-v" in sys.argv)
    print(LIB)
