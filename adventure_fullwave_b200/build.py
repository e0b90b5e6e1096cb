"""Builds the CUDA library ``libfwgpu.so`` in-tree for sm_100a.

The library holds the C ABI declared in ``include/fwgpu.h``.  The element
kernel is compiled with floating-point contraction off so its arithmetic
matches the reference's bit for bit; the other kernels use the default.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libfwgpu.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = [
    ("fw_element.cu", ["-fmad=false"]),
    ("fw_kernels.cu", []),
    ("fw_multi.cu", []),
    ("fw_capi.cu", []),
    ("fw_noalloc.cu", []),
    ("fw_build.cpp", []),
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(out: str, deps) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    """Compile every source to an object under csrc/_build and link the
    shared library next to this file.  Returns the library path."""
    bdir = os.path.join(CSRC, "_build")
    os.makedirs(bdir, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(HERE, "..", "include", "fwgpu.h"))
    objs = []
    for src, extra in SOURCES:
        sp = os.path.join(CSRC, src)
        op = os.path.join(bdir, src + ".o")
        objs.append(op)
        if not force and not _stale(op, [sp] + headers):
            continue
        cmd = [nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-c", sp, "-o", op, *extra]
        if src.endswith(".cpp"):
            cmd[1:1] = ["-x", "cu"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lcudart", "-ldl"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv))
