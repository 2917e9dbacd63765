"""Builds ``montepath_b200/lib/libmontepath_cuda.so`` for sm_100a with nvcc.

Usage: ``python -m montepath_b200.build`` (or ``__graft_entry__.build()``).
The three translation units compile in parallel and link into one shared
library with the CUDA runtime linked statically, so the library loads on a
machine without a GPU (calls then return MPC_E_NO_DEVICE).
"""

from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "lib")
OBJ_DIR = os.path.join(OUT_DIR, "obj")
LIBRARY = os.path.join(OUT_DIR, "libmontepath_cuda.so")
SOURCES = ["mpc_kernels.cu", "mpc_runtime.cu", "mpc_server.cu", "mpc_peaks.cu", "mpc_noalloc.cu", "mpc_greeks.cu", "mpc_merton.cu"]
HEADERS = [
    "mpc_device.cuh",
    "mpc_launch.h",
    "mpc_runtime.h",
    "mpc_types.h",
    "sobol_directions.h",
    os.path.join("..", "..", "include", "montepath_cuda.h"),
]

NVCC_FLAGS = [
    "-gencode",
    "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "-O3",
    "-std=c++17",
    "-Xcompiler",
    "-fPIC,-O2",
    "-Xptxas",
    "-warn-spills",
]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build the backend")
    return path


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str) -> str:
    obj = os.path.join(OBJ_DIR, os.path.splitext(src)[0] + ".o")
    deps = [os.path.join(CSRC, src)] + [os.path.join(CSRC, h) for h in HEADERS]
    if _stale(obj, deps):
        cmd = [nvcc(), *NVCC_FLAGS, "-c", os.path.join(CSRC, src), "-o", obj]
        subprocess.run(cmd, check=True)
    return obj


def build(force: bool = False, verbose: bool = True) -> str:
    os.makedirs(OBJ_DIR, exist_ok=True)
    if force:
        for f in os.listdir(OBJ_DIR):
            os.remove(os.path.join(OBJ_DIR, f))
    with concurrent.futures.ThreadPoolExecutor(max_workers=len(SOURCES)) as pool:
        objs = list(pool.map(_compile, SOURCES))
    if force or _stale(LIBRARY, objs):
        cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIBRARY, *objs, "-lpthread"]
        subprocess.run(cmd, check=True)
    if verbose:
        print(f"built {LIBRARY}", file=sys.stderr)
    return LIBRARY


if __name__ == "__main__":
    build(force="--force" in sys.argv)
