"""Build libbimp_b200.so (sm_100a) in-tree with nvcc.

    python cuda-bimp_b200/build.py            # library
    python cuda-bimp_b200/build.py --force    # rebuild everything

Objects go to cuda-bimp_b200/_build/, the library to cuda-bimp_b200/lib/.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
BUILD = PKG / "_build"
LIB = PKG / "lib" / "libbimp_b200.so"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              f"-I{INCLUDE}", f"-I{CSRC}"]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", f"-I{INCLUDE}", f"-I{CSRC}", "-I/usr/local/cuda/include"]

SOURCES = [
    ("bank.cpp", "cxx"),
    ("kernels.cu", "cuda"),
    ("capi.cu", "cuda"),
    ("noalloc.cu", "cuda"),
    ("extras.cu", "cuda"),
    ("adjoint.cu", "cuda"),
]
HEADERS = sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))


def _stale(out: Path, deps) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def _run(cmd):
    print(" ".join(str(c) for c in cmd), flush=True)
    subprocess.run([str(c) for c in cmd], check=True)


def build(force: bool = False, verbose_ptxas: bool = False) -> Path:
    BUILD.mkdir(parents=True, exist_ok=True)
    LIB.parent.mkdir(parents=True, exist_ok=True)
    objs = []
    for src, kind in SOURCES:
        s = CSRC / src
        o = BUILD / (src + ".o")
        objs.append(o)
        if force or _stale(o, [s, *HEADERS]):
            if kind == "cuda":
                extra = ["-Xptxas", "-v"] if verbose_ptxas else []
                _run([NVCC, *ARCH, *CUDA_FLAGS, *extra, "-c", s, "-o", o])
            else:
                _run(["g++", *CXX_FLAGS, "-c", s, "-o", o])
    if force or _stale(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart_static", "-ldl", "-lrt", "-lpthread"])
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print register/smem usage")
    a = ap.parse_args()
    build(force=a.force, verbose_ptxas=a.ptxas)
    sys.exit(0)
