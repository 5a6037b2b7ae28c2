"""Builds ``libsofia_nb.so`` (all CUDA kernels + the C ABI) for sm_100a, in tree.

Each ``csrc/*.cu`` translation unit is compiled with
``-gencode arch=compute_100a,code=sm_100a -fmad=false``: the compiler contracts
no product into a later sum, so every real*4 / real*8 operation is rounded
separately, in source order, and the fused multiply-adds that the kernels want
are written out (``__fma_rn``, ``__fmaf_rn``, ``__ffma2_rn``).  A kernel body
then gives the same bits whichever kernel inlines it: the single-system
kernels and the batched ones that run the same bodies for many replicas
produce identical trajectories.
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libsofia_nb.so")
INCLUDE = os.path.join(os.path.dirname(PKG), "include")

NVCC = os.environ.get("SOFIA_NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
          "-ccbin", "g++"]


def _units():
    return sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    return hs


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, extra_flags: list[str] | None = None) -> str:
    os.makedirs(OBJ, exist_ok=True)
    headers = _headers()
    objs = []
    env = dict(os.environ)
    env.pop("CC", None)
    env.pop("CXX", None)
    for u in _units():
        src = os.path.join(CSRC, u)
        obj = os.path.join(OBJ, u[:-3] + ".o")
        objs.append(obj)
        if not _stale(obj, [src] + headers + [__file__]):
            continue
        flags = list(COMMON) + ARCH + ["-fmad=false"] + (extra_flags or [])
        cmd = [NVCC] + flags + ["-I", INCLUDE, "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True, env=env)
    if _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcuda"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True, env=env)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True))
