"""Build libmycel_b200.so in-tree with nvcc for sm_100a (cross-compiles without a GPU).

fp64_kernels.cu is compiled with -fmad=false: the plain FP64 path must round every product and sum separately,
as the reference's RyuJIT code does. The other translation units use the default (FMA allowed).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmycel_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off", "--expt-relaxed-constexpr",
          "-I", os.path.join(HERE, "..", "include")]

UNITS = [
    ("fp64_kernels.cu", ["-fmad=false"]),
    ("fp32_kernels.cu", ["-fmad=true"]),
    ("api.cu", ["-fmad=true"]),
    ("simp.cu", ["-fmad=true"]),
    ("hex8.cpp", []),
    ("server.cpp", []),
    ("surface_nets.cu", ["-fmad=false"]),
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


def build(verbose: bool = False, force: bool = False, extra=None) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in ("internal.h", "libm_pow.h", "libm_pow_tables.h")]
    headers.append(os.path.join(HERE, "..", "include", "mycel.h"))
    objs = []
    for src, flags in UNITS:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if force or _stale(obj, [path] + headers):
            cmd = [nvcc()] + ARCH + COMMON + flags + (extra or []) + ["-c", path, "-o", obj]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.check_call(cmd)
    if force or _stale(LIB, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else None)
