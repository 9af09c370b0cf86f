"""Builds libcn_physics.so (the sm_100a substep library) in-tree.

Usage: python cressim-neo_b200/build.py [--force]

Every CUDA translation unit is compiled for sm_100a only, with --fmad=false so float32
results follow the reference's expression order exactly (see csrc/cn_math.cuh).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
INCLUDE = HERE.parent / "include"
LIB = HERE / "libcn_physics.so"
OBJ_DIR = HERE / "_build"

CUDA_SOURCES = ["cn_kernels.cu", "cn_sort.cu", "cn_noalloc.cu", "cn_diff.cu", "cn_rigid.cu"]
HOST_SOURCES = ["cn_solver.cpp", "cn_world.cpp", "cn_batch.cpp", "cn_server.cpp"]
HEADERS = ["cn_device.h", "cn_math.cuh", "cn_internal.h"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "--fmad=false", "-prec-div=true", "-prec-sqrt=true",
    "-Xcompiler", "-fPIC,-fvisibility=hidden,-ffp-contract=off",
]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(path).exists():
        raise RuntimeError("nvcc not found; the CUDA 12.9 toolkit is required to build libcn_physics.so")
    return path


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.exists() and d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    OBJ_DIR.mkdir(exist_ok=True)
    headers = [CSRC / h for h in HEADERS] + [INCLUDE / "cn_physics.h"]
    objs = []
    for src in CUDA_SOURCES + HOST_SOURCES:
        s = CSRC / src
        if not s.exists():
            continue
        o = OBJ_DIR / (s.stem + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            lang = ["-x", "cu"] if s.suffix == ".cu" else ["-x", "c++"]
            cmd = [nvcc(), *NVCC_FLAGS, *lang, "-I", str(INCLUDE), "-c", str(s), "-o", str(o)]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", str(LIB),
               *map(str, objs), "-Xcompiler", "-fPIC"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
