"""Build libptychox (the C-ABI CUDA library) in-tree for sm_100a.

``python -m ptychox_b200.build`` compiles every ``csrc/*.cu`` translation unit with nvcc
(in parallel) and links ``ptychox_b200/_lib/libptychox.so``.  The library is rebuilt
only when a source or header is newer than it (``force=True`` rebuilds always).
"""

from __future__ import annotations

import concurrent.futures as _cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIBDIR = PKG / "_lib"
LIBNAME = "libptychox.so"
INCLUDE = PKG.parent / "include"

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3"]


def _nvcc() -> str:
    cand = shutil.which("nvcc")
    if cand:
        return cand
    home = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    path = Path(home) / "bin" / "nvcc"
    if path.exists():
        return str(path)
    raise RuntimeError("nvcc not found (set CUDA_HOME)")


def library_path() -> Path:
    return LIBDIR / LIBNAME


def _sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _headers() -> list[Path]:
    return sorted(list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(INCLUDE.glob("*.h")))


def needs_build() -> bool:
    lib = library_path()
    if not lib.exists():
        return True
    stamp = lib.stat().st_mtime
    return any(p.stat().st_mtime > stamp for p in _sources() + _headers())


def _compile_one(nvcc: str, src: Path, obj: Path, verbose: bool) -> None:
    cmd = [nvcc, *ARCH_FLAGS, *COMMON_FLAGS, "-I", str(INCLUDE), "-c", str(src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n{res.stdout}\n{res.stderr}")


def build_library(force: bool = False, verbose: bool = False) -> Path:
    """Compile and link libptychox.so; returns its path."""
    lib = library_path()
    if not force and not needs_build():
        return lib
    nvcc = _nvcc()
    objdir = LIBDIR / "obj"
    objdir.mkdir(parents=True, exist_ok=True)
    srcs = _sources()
    objs = [objdir / (s.stem + ".o") for s in srcs]
    workers = min(len(srcs), max(1, os.cpu_count() or 1))
    with _cf.ThreadPoolExecutor(max_workers=workers) as ex:
        futs = [ex.submit(_compile_one, nvcc, s, o, verbose) for s, o in zip(srcs, objs)]
        for f in futs:
            f.result()
    tmp = lib.with_suffix(".so.tmp")
    cmd = [nvcc, *ARCH_FLAGS, "-shared", "-o", str(tmp), *[str(o) for o in objs], "-lcudart"]
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    os.replace(tmp, lib)
    return lib


if __name__ == "__main__":
    path = build_library(force="--force" in sys.argv, verbose=True)
    print(path)
