"""Build libmbirgpu.so in-tree for sm_100a with nvcc.

``python -m phasecon_b200.build`` (or ``build()``) compiles every CUDA and C++
source under phasecon_b200/csrc into phasecon_b200/libmbirgpu.so. Objects go
to phasecon_b200/_build/. nvcc cross-compiles for sm_100a without a GPU.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
OUT = os.path.join(PKG, "libmbirgpu.so")
BUILD = os.path.join(PKG, "_build")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off", "-I", CSRC,
          "-I", os.path.join(os.path.dirname(PKG), "include")]
# files whose double-precision geometry must round like the reference
NO_FMA = {"kernels_amatrix.cu", "pc_simulate.cu"}


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources() -> list[str]:
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def _compile(src: str) -> str:
    nvcc = _nvcc()
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(
            os.path.getmtime(p) for p in [src] + [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith(".h")]
            + [os.path.join(os.path.dirname(PKG), "include", "mbirgpu.h")]):
        return obj
    cmd = [nvcc] + ARCH + COMMON + ["-c", src, "-o", obj]
    if os.path.basename(src) in NO_FMA:
        cmd.insert(1, "-fmad=false")
    subprocess.run(cmd, check=True)
    return obj


def build(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(_compile, srcs))
    newest = max(os.path.getmtime(o) for o in objs)
    if not os.path.exists(OUT) or os.path.getmtime(OUT) < newest:
        cmd = [_nvcc()] + ARCH + ["-shared", "-o", OUT] + objs + ["-lcudart"]
        subprocess.run(cmd, check=True)
    if verbose:
        print("built", OUT)
    return OUT


if __name__ == "__main__":
    build(verbose=True)
