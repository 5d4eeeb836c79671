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
# gpu_backend_kb.cu / capi_field_kb.cu recompile gpu_backend.cu / capi_field.cu
# for KoalaBear^4 (QF_FIELD_KB); the others are F65521^8 or field-independent.
SOURCES = [PKG / "csrc" / n for n in ("capi.cu", "gpu_common.cu", "gpu_backend.cu", "capi_field.cu", "noalloc.cu",
                                      "intpeak.cu", "gpu_backend_kb.cu", "capi_field_kb.cu")]
OBJ_DIR = PKG / "_build"
HEADERS = sorted((PKG / "csrc").rglob("*.h")) + sorted((PKG / "csrc").rglob("*.cuh"))

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC,-fopenmp,-O2,-ffp-contract=off",
    "--expt-relaxed-constexpr",
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
    """Compiles each source to an object (in parallel), then links the library."""
    if not force and not stale():
        return LIB
    from concurrent.futures import ThreadPoolExecutor

    LIB_DIR.mkdir(exist_ok=True)
    OBJ_DIR.mkdir(exist_ok=True)

    def compile_one(src: Path) -> Path:
        obj = OBJ_DIR / (src.stem + ".o")
        cmd = [nvcc(), *NVCC_FLAGS, "-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        return obj

    with ThreadPoolExecutor(max_workers=min(len(SOURCES), os.cpu_count() or 1)) as pool:
        objs = list(pool.map(compile_one, SOURCES))
    cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", *map(str, objs), "-o", str(LIB), "-lgomp"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
