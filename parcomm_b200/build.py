"""Builds libparcomm_qafold.so for sm_100a with nvcc (in-tree, no JIT cache).

Usage: python -m parcomm_b200.build   (or parcomm_b200.build.build())
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_DIR = PKG / "_lib"
LIB = LIB_DIR / "libparcomm_qafold.so"
SOURCES = [PKG / "csrc" / "capi.cu", PKG / "csrc" / "gpu_backend.cu", PKG / "csrc" / "noalloc.cu"]
HEADERS = sorted((PKG / "csrc").rglob("*.h")) + sorted((PKG / "csrc").rglob("*.cuh"))

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC,-fopenmp,-O2,-ffp-contract=off",
    "--expt-relaxed-constexpr",
    "-shared",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or Path(cand).exists()):
            return cand
    return "nvcc"


def stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    return any(p.stat().st_mtime > t for p in SOURCES + HEADERS + [PKG.parent / "include" / "parcomm_qafold.h"])


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not stale():
        return LIB
    LIB_DIR.mkdir(exist_ok=True)
    cmd = [nvcc(), *NVCC_FLAGS, *map(str, SOURCES), "-o", str(LIB), "-lgomp"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
