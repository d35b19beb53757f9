"""Builds the in-tree CUDA library brae_b200/libbrae_gamg.so for sm_100a with nvcc.

    python -m brae_b200.build          # incremental (objects in brae_b200/_build/)

Every kernel is compiled for sm_100a only, with --fmad=false: the parity kernels must round each
product and each sum separately, as the reference's x86-64 host loops do.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libbrae_gamg.so")
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
SOURCES = ["hierarchy.cu", "solver.cu", "capi.cu", "server.cu", "batch.cu", "pair.cu", "pipe.cu", "items.cu", "assemble.cu"]
FLAGS = ["-std=c++17", "-O3", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
         "--fmad=false", "-Xcompiler", "-fPIC,-fvisibility=hidden,-ffp-contract=off", "-Xptxas", "-O3"]


def _deps(src: str) -> list[str]:
    hdrs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    return [os.path.join(CSRC, src), os.path.join(HERE, "..", "include", "brae_gamg.h")] + hdrs


def _stale(obj: str, deps: list[str]) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(BUILD, src.replace(".cu", ".o"))
    if _stale(obj, _deps(src)):
        cmd = [NVCC, *FLAGS, "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
        noise = [ln for ln in r.stderr.splitlines() if ln.strip() and "compute_" not in ln]
        if noise and verbose:
            print("\n".join(noise))
    return obj


def build(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), SOURCES))
    if not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objs, "-o", LIB]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-q" not in sys.argv))
