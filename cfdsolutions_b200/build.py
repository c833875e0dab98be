"""Build the in-tree CUDA library ``cfdsolutions_b200/_lib/libcfd_b200.so``.

Every translation unit is compiled by nvcc for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a``) with ``-lineinfo``; the result
lives inside the package so it travels with the source tree.  Run as
``python cfdsolutions_b200/build.py`` (as a script, so the stale library is not
loaded by the package import first) or call :func:`build`.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
OUT_DIR = PKG / "_lib"
LIB = OUT_DIR / "libcfd_b200.so"
OBJ_DIR = PKG / "_build"

CU_SOURCES = ["core.cu", "gradient.cu", "linsolve.cu", "ilu_mc.cu", "gs_static.cu", "serve.cu", "fd_jacobian.cu"]
# per-file nvcc flags: the finite-difference Jacobian must round every
# expression as written (no fused multiply-add) to reproduce the reference
FILE_FLAGS = {"fd_jacobian.cu": ["-fmad=false"]}
CXX_SOURCES = ["mesh.cpp", "vtk.cpp", "rmsio.cpp"]
HEADERS = ["cfd_internal.h", "host_par.h", "ctx.cuh", "kernels.cuh", "physics.cuh", "ilu_mc.cuh"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-Xptxas", "-O3"]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-pthread", "-Wall", "-Wno-unused-function"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found (set NVCC)")


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> Path:
    """Compile (incrementally) and link the library; returns its path."""
    OUT_DIR.mkdir(exist_ok=True)
    OBJ_DIR.mkdir(exist_ok=True)
    nvcc = _nvcc()
    include = ["-I", str(CSRC), "-I", str(PKG.parent / "include")]
    headers = [CSRC / h for h in HEADERS] + [PKG.parent / "include" / "cfd_b200.h"]
    objs = []
    for src in CU_SOURCES:
        s = CSRC / src
        o = OBJ_DIR / (src + ".o")
        if force or _stale(o, [s, *headers]):
            cmd = [nvcc, *ARCH, *NVCC_FLAGS, *FILE_FLAGS.get(src, []), *include, "-c", str(s), "-o", str(o)]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
        objs.append(o)
    for src in CXX_SOURCES:
        s = CSRC / src
        o = OBJ_DIR / (src + ".o")
        if force or _stale(o, [s, *headers]):
            cmd = ["g++", *CXX_FLAGS, *include, "-c", str(s), "-o", str(o)]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
        objs.append(o)
    if force or _stale(LIB, objs):
        cmd = [nvcc, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
    print(LIB)
