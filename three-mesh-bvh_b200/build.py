"""Build recipe for libbvhcuda.so (nvcc, sm_100a), written next to this file.

The library is built in-tree so that it travels with the repository; nothing is installed into
site-packages and nothing is JIT-compiled at import time.  Each source compiles to its own object
(in parallel, under _build/, rebuilt when the source or any header changed), then one link.
"""
from __future__ import annotations

import os
import subprocess
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
LIB = PKG / "libbvhcuda.so"
OBJ_DIR = PKG / "_build"
CSRC = PKG / "csrc"
SOURCES = [CSRC / n for n in ("api.cu", "kernels_first.cu", "kernels_packet.cu", "kernels_all.cu", "kernels_query.cu", "kernels_scene.cu",
                              "adjoint.cu", "noalloc.cu", "raysort.cu", "refit.cu", "gpubuild.cu", "autotune.cu",
                              "builder.cpp")]
HEADERS = [ROOT / "include" / "bvhcuda.h"] + sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh"))

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [*ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3"]


def nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def _obj(src: Path) -> Path:
    return OBJ_DIR / (src.name + ".o")


def _stale(src: Path, newest_header: float) -> bool:
    o = _obj(src)
    return not o.exists() or o.stat().st_mtime < max(src.stat().st_mtime, newest_header)


def needs_build() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    return any(p.stat().st_mtime > t for p in SOURCES + HEADERS)


def _compile(src: Path, verbose: bool) -> subprocess.CompletedProcess:
    cmd = [nvcc(), *NVCC_FLAGS, f"-I{ROOT / 'include'}", f"-I{CSRC}", "-c", str(src), "-o", str(_obj(src))]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    return subprocess.run(cmd, capture_output=True, text=True)


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not needs_build():
        return LIB
    OBJ_DIR.mkdir(exist_ok=True)
    newest = max(p.stat().st_mtime for p in HEADERS)
    todo = [s for s in SOURCES if force or _stale(s, newest)]
    # the largest units first, so that the longest compile starts at once
    todo.sort(key=lambda p: -p.stat().st_size)
    with ThreadPoolExecutor(max_workers=max(1, min(len(todo), os.cpu_count() or 1))) as ex:
        results = list(ex.map(lambda s: (s, _compile(s, verbose)), todo))
    for src, res in results:
        if res.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src.name} ({res.returncode}):\n{res.stdout}\n{res.stderr}")
        if verbose:
            print(src.name, res.stderr)
    link = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, map(_obj, SOURCES))]
    res = subprocess.run(link, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc link failed ({res.returncode}):\n{res.stdout}\n{res.stderr}")
    return LIB


if __name__ == "__main__":
    import sys

    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
