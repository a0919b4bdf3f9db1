"""Build the sm_100a shared library ``tensorsph_b200/_lib/libtsph_b200.so``.

    python -m tensorsph_b200.build          # incremental
    python -m tensorsph_b200.build --force  # rebuild everything

Every ``csrc/*.cu`` file is compiled to an object with
``-gencode arch=compute_100a,code=sm_100a`` (cross-compiles on a host without
a GPU) and linked into one shared library loaded through ctypes.  No JIT cache
is involved, so the built file travels with the source tree.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
from pathlib import Path
import shutil
import subprocess
import sys

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
OUT_DIR = PKG / "_lib"
OBJ_DIR = PKG / "_build"
LIB = OUT_DIR / "libtsph_b200.so"
INCLUDE = PKG.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-Xptxas", "-warn-spills"]


def nvcc() -> str:
    found = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(found).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libtsph_b200")
    return found


def _deps_mtime() -> float:
    headers = list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    return max((p.stat().st_mtime for p in headers), default=0.0)


def _compile(src: Path, force: bool, verbose_ptxas: bool) -> Path:
    obj = OBJ_DIR / (src.stem + ".o")
    if (not force and obj.exists() and obj.stat().st_mtime >= src.stat().st_mtime
            and obj.stat().st_mtime >= _deps_mtime()):
        return obj
    cmd = [nvcc(), *ARCH, *FLAGS, "-I", str(INCLUDE), "-c", str(src), "-o", str(obj)]
    if verbose_ptxas:
        cmd[1:1] = ["-Xptxas", "-v"]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{proc.stderr}")
    if verbose_ptxas and proc.stderr:
        sys.stderr.write(proc.stderr)
    return obj


def build(force: bool = False, verbose_ptxas: bool = False) -> Path:
    OUT_DIR.mkdir(exist_ok=True)
    OBJ_DIR.mkdir(exist_ok=True)
    sources = sorted(CSRC.glob("*.cu"))
    workers = max(1, min(len(sources), os.cpu_count() or 1))
    with cf.ThreadPoolExecutor(workers) as pool:
        objs = list(pool.map(lambda s: _compile(s, force, verbose_ptxas), sources))
    newest = max(o.stat().st_mtime for o in objs)
    if force or not LIB.exists() or LIB.stat().st_mtime < newest:
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lcudart"]
        proc = subprocess.run(cmd, capture_output=True, text=True)
        if proc.returncode != 0:
            raise RuntimeError(f"link failed:\n{proc.stderr}")
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print -Xptxas -v resource usage")
    args = ap.parse_args()
    print(build(force=args.force, verbose_ptxas=args.ptxas))
