"""Builds libtopo.so (the sm_100a C-ABI library) in-tree with nvcc.

    python build.py            # incremental
    python build.py --force    # rebuild everything
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libtopo.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
         "--expt-relaxed-constexpr", "-I", INCLUDE]

SOURCES = ["setup.cpp", "serve.cpp", "kernels_elem.cu", "amg.cu", "solver.cu", "mma.cu", "abi.cu", "noalloc.cu", "block.cu", "block_solve.cu", "stepgraph.cu"]
HEADERS = ["common.cuh", "ctx.h"]


def _stale(obj: str, src: str) -> bool:
    if not os.path.exists(obj):
        return True
    deps = [src] + [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "topo.h")]
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _compile(src: str, force: bool, extra: list[str]) -> str:
    path = os.path.join(CSRC, src)
    obj = os.path.join(BUILD, src.rsplit(".", 1)[0] + ".o")
    if force or _stale(obj, path):
        lang = ["-x", "cu"] if src.endswith(".cu") else ["-x", "c++"]
        cmd = [NVCC] + ARCH + FLAGS + extra + lang + ["-c", path, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
        if r.stderr.strip():
            sys.stderr.write(r.stderr)
    return obj


def build(force: bool = False, verbose_ptxas: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    extra = ["-Xptxas", "-v"] if verbose_ptxas else []
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, extra), SOURCES))
    if force or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    # the main.cpp-shaped driver program over the C++ classes (include/topopt.hpp)
    exe = os.path.join(HERE, "topopt")
    src = os.path.join(HERE, "host", "topopt_main.cpp")
    hdrs = [os.path.join(INCLUDE, h) for h in ("topo.h", "topopt.hpp")]
    if force or not os.path.exists(exe) or any(os.path.getmtime(p) > os.path.getmtime(exe) for p in [src, LIB] + hdrs):
        cmd = ["g++", "-O2", "-std=c++17", "-I", INCLUDE, src, "-L", HERE, "-ltopo", "-Wl,-rpath,$ORIGIN",
               "-o", exe]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"topopt build failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose_ptxas="--ptxas" in sys.argv))
