"""Build libfastwigner.so in-tree with nvcc for sm_100a.

Usage: ``python -m fastwigner_b200.build [--verbose]``.  The library is
written next to this file (``fastwigner_b200/libfastwigner.so``) so that it
travels with the source tree; it is rebuilt only when a source is newer.
"""
from __future__ import annotations

import os
import re
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
LIB = PKG / "libfastwigner.so"
BUILD = PKG / "_build"

SOURCES = [
    "api.cu",
    "wigner_passes.cu",
    "wigner_colp.cu",
    "wigner_rowp.cu",
    "wigner_generic.cu",
    "rho_api.cu",
    "expr.cu",
    "fno.cu",
    "fno_umma.cu",
    "batch.cu",
]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]


def _nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def _sources() -> list[Path]:
    return [CSRC / s for s in SOURCES if (CSRC / s).exists()]


_INCLUDE_RE = re.compile(r'^\s*#\s*include\s+"([^"]+)"', re.M)


def _deps(src: Path) -> set[Path]:
    """src and every file it pulls in with #include "..." (recursively, any
    extension: the translation units include .cu files as well as headers)."""
    seen: set[Path] = set()
    todo = [src.resolve()]
    while todo:
        f = todo.pop()
        if f in seen or not f.exists():
            continue
        seen.add(f)
        for name in _INCLUDE_RE.findall(f.read_text(errors="replace")):
            for base in (f.parent, INCLUDE):
                cand = (base / name).resolve()
                if cand.exists():
                    todo.append(cand)
                    break
    return seen


def _stale(obj: Path, src: Path) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(d.stat().st_mtime > t for d in _deps(src))


def build(verbose: bool = False, force: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    objs = []
    nvcc = _nvcc()
    jobs = []
    for src in _sources():
        obj = BUILD / (src.stem + ".o")
        objs.append(obj)
        if force or _stale(obj, src):
            cmd = [nvcc, *ARCH, *NVCC_FLAGS, "-I", str(INCLUDE), "-c", str(src), "-o", str(obj)]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
                print(" ".join(cmd), flush=True)
            jobs.append(cmd)
    # the translation units are independent: compile them concurrently
    workers = max(1, min(len(jobs), os.cpu_count() or 1))
    with ThreadPoolExecutor(max_workers=workers) as ex:
        for f in [ex.submit(subprocess.run, cmd, check=True) for cmd in jobs]:
            f.result()
    if force or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        cmd = [nvcc, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart", "-lnvrtc"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, force="--force" in sys.argv)
    print(LIB)
