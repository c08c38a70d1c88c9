"""Build recipe of the native library cirrus_b200/_lib/libcirrus_b200.so (sm_100a only).

Compiles the CUDA/C++ sources of cirrus_b200/csrc with nvcc for
`-gencode arch=compute_100a,code=sm_100a -lineinfo` and links one shared library exporting
the C ABI declared in include/cirrus_b200.h.  The library is built in-tree so it travels
with the repository to the GPU machine; nothing is JIT-compiled at import time.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIBDIR = PKG / "_lib"
LIB = LIBDIR / "libcirrus_b200.so"
INCLUDE = PKG.parent / "include"

GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", *GENCODE, "-Xcompiler", "-fPIC,-fopenmp,-O3",
              "-I", str(CSRC), "-I", str(INCLUDE)]
SOURCES = ["topology.cpp", "grid.cu", "kernels.cu", "lap_tma.cu", "lap8.cu", "amg.cu", "vcycle_fused.cu", "rhs.cu", "interop.cu", "solver.cu", "capi.cu", "noalloc.cu", "autotune.cu", "serve.cpp", "holder.cpp", "dtopo.cu"]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(path).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build cirrus_b200")
    return path


def _newest_source_mtime() -> float:
    files = list(CSRC.glob("*")) + [INCLUDE / "cirrus_b200.h", Path(__file__)]
    return max(f.stat().st_mtime for f in files if f.is_file())


def needs_build() -> bool:
    return not LIB.exists() or LIB.stat().st_mtime < _newest_source_mtime()


def build(force: bool = False, verbose: bool = False, extra_flags: list[str] | None = None) -> Path:
    if not force and not needs_build():
        return LIB
    LIBDIR.mkdir(exist_ok=True)
    objdir = LIBDIR / "obj"
    objdir.mkdir(exist_ok=True)
    cc = nvcc()
    flags = NVCC_FLAGS + list(extra_flags or [])

    def compile_one(src: str) -> Path:
        obj = objdir / (src + ".o")
        lang = ["-x", "cu"] if src.endswith(".cu") else []
        cmd = [cc, *flags, *lang, "-c", str(CSRC / src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{res.stdout}\n{res.stderr}")
        return obj

    with ThreadPoolExecutor(max_workers=min(len(SOURCES), os.cpu_count() or 4)) as ex:
        objs = list(ex.map(compile_one, SOURCES))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [cc, "-shared", *GENCODE, "-Xcompiler", "-fPIC,-fopenmp", *map(str, objs), "-o", str(tmp), "-lgomp"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
