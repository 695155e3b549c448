"""Build recipe for libbvhcuda.so (nvcc, sm_100a), written next to this file.

The library is built in-tree so that it travels with the repository; nothing is installed into
site-packages and nothing is JIT-compiled at import time.
"""
from __future__ import annotations

import os
import subprocess
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
LIB = PKG / "libbvhcuda.so"
SOURCES = [PKG / "csrc" / "api.cu", PKG / "csrc" / "kernels.cu", PKG / "csrc" / "adjoint.cu", PKG / "csrc" / "noalloc.cu",
           PKG / "csrc" / "raysort.cu", PKG / "csrc" / "refit.cu", PKG / "csrc" / "gpubuild.cu",
           PKG / "csrc" / "builder.cpp"]
HEADERS = [ROOT / "include" / "bvhcuda.h"] + sorted((PKG / "csrc").glob("*.h")) + sorted((PKG / "csrc").glob("*.cuh"))

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
    "-shared",
]


def nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def needs_build() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    return any(p.stat().st_mtime > t for p in SOURCES + HEADERS)


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not needs_build():
        return LIB
    cmd = [nvcc(), *NVCC_FLAGS, f"-I{ROOT / 'include'}", f"-I{PKG / 'csrc'}", "-o", str(LIB), *map(str, SOURCES)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed ({res.returncode}):\n{res.stdout}\n{res.stderr}")
    if verbose:
        print(res.stderr)
    return LIB


if __name__ == "__main__":
    import sys

    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
